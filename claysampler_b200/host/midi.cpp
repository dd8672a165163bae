// Standard MIDI File reader producing frame-timed events, following the
// reference's src/io/midi.cpp: format 0/1 with PPQ timing, a tempo map, the
// `natural` performance preparation (pedal-extended end, ClayEngine controller
// defaults) and the frame rounding of src/io/midi.cpp:255-297.
#include "host_types.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <iterator>
#include <limits>
#include <stdexcept>
#include <string_view>

namespace csh {
namespace {

class Reader {
public:
    explicit Reader(std::string_view bytes) : rest_(bytes) {}
    bool empty() const { return rest_.empty(); }

    std::string_view take(size_t count)
    {
        if (count > rest_.size())
            throw std::runtime_error("truncated MIDI");
        const auto out = rest_.substr(0, count);
        rest_.remove_prefix(count);
        return out;
    }

    int byte() { return static_cast<unsigned char>(take(1)[0]); }

    uint32_t bigEndian(int width)
    {
        uint32_t value = 0;
        for (int i = 0; i < width; ++i)
            value = (value << 8) | uint32_t(byte());
        return value;
    }

    uint32_t varLen()
    {
        uint32_t value = 0;
        for (int i = 0; i < 4; ++i) {
            const int b = byte();
            value = (value << 7) | uint32_t(b & 0x7f);
            if (b < 0x80)
                return value;
        }
        throw std::runtime_error("invalid MIDI variable-length value");
    }

private:
    std::string_view rest_;
};

struct Message {
    uint64_t tick;
    int status, a, b;                   // status 0xff: tempo in a; status 0: end of track
};

void readTrack(Reader track, std::vector<Message>& out)
{
    uint64_t tick = 0;
    int running = 0;
    while (!track.empty()) {
        tick += track.varLen();
        int status = track.byte();
        int first = -1;
        if (status < 0x80) {
            first = status;
            status = running;
            if (!status)
                throw std::runtime_error("MIDI running status has no channel message");
        }
        if (status == 0xff) {
            const int type = track.byte();
            Reader meta(track.take(track.varLen()));
            if (type == 0x51) {
                const uint32_t tempo = meta.bigEndian(3);
                if (!tempo || !meta.empty())
                    throw std::runtime_error("invalid MIDI tempo");
                out.push_back({tick, 0xff, int(tempo), 0});
            } else if (type == 0x2f) {
                if (!meta.empty())
                    throw std::runtime_error("invalid MIDI end-of-track");
                out.push_back({tick, 0, 0, 0});
                return;
            }
            running = 0;
            continue;
        }
        if (status >= 0xf0)
            throw std::runtime_error("unsupported MIDI system or SysEx message");
        running = status;
        const int a = first < 0 ? track.byte() : first;
        const int kind = status >> 4;
        const int b = (kind == 0xc || kind == 0xd) ? 0 : track.byte();
        if (a >= 128 || b >= 128)
            throw std::runtime_error("invalid MIDI data byte");
        out.push_back({tick, status, a, b});
    }
    throw std::runtime_error("missing MIDI end-of-track");
}

int order(const Message& m)
{
    const int kind = m.status >> 4;
    if (kind == 9 && m.b != 0)
        return 30;
    if (kind == 8 || kind == 9)
        return 25;
    return 15;
}

// The natural-tail performance (src/io/midi.cpp:115-175): ends at the last complete
// note or a later pedal release, drops volume/pan/bank/effect controllers and
// trailing panic commands, sets CC7=100 and CC10=64, and releases the pedals at
// the end.
void prepareNatural(std::vector<Message>& messages)
{
    std::array<std::array<int, 128>, 16> held{};
    uint64_t lastNote = 0;
    int channel = -1;
    for (const auto& m : messages) {
        const int kind = m.status >> 4;
        if (kind != 8 && kind != 9)
            continue;
        const int current = m.status & 15;
        int& count = held[size_t(current)][size_t(m.a)];
        if (kind == 9 && m.b) {
            ++count;
        } else if (count > 0) {
            --count;
            if (channel >= 0 && channel != current)
                throw std::runtime_error("multiple MIDI channels in one render job");
            channel = current;
            lastNote = m.tick;
        }
    }
    if (channel < 0)
        throw std::runtime_error("natural rendering requires a complete MIDI note");
    constexpr int pedals[] = {64, 66, 69};
    std::array<bool, 3> down{};
    uint64_t end = lastNote;
    for (const auto& m : messages) {
        if ((m.status >> 4) != 0xb)
            continue;
        for (size_t p = 0; p < down.size(); ++p) {
            if (m.a != pedals[p])
                continue;
            if (m.tick <= end)
                down[p] = m.b >= 64;
            else if (down[p] && m.b < 64) {
                end = m.tick;
                down[p] = false;
            }
        }
    }
    messages.erase(std::remove_if(messages.begin(), messages.end(), [&](const Message& m) {
        if (!m.status || m.tick > end || (m.status >> 4) == 0xc)
            return true;
        if ((m.status >> 4) != 0xb)
            return false;
        switch (m.a) {
        case 0: case 7: case 10: case 32: case 91: case 93: return true;
        case 120: case 123: return m.tick >= lastNote;
        default: return false;
        }
    }), messages.end());
    const int control = 0xb0 | channel;
    messages.insert(messages.begin(), {{0, control, 7, 100}, {0, control, 10, 64}});
    std::stable_sort(messages.begin(), messages.end(), [](const Message& x, const Message& y) {
        return x.tick == y.tick ? order(x) < order(y) : x.tick < y.tick;
    });
    for (int cc : pedals)
        messages.push_back({end, control, cc, 0});
    messages.push_back({end, 0, 0, 0});
}

// Onsets and body length for the quality gate (src/io/midi.cpp:177-216).
void measureBody(const std::vector<Message>& messages, int rate, int division, Midi& midi)
{
    struct Pending { int start, next; };
    std::vector<Pending> pending{{0, 0}};
    std::vector<int> head(16 * 128, 0), tail(16 * 128, 0);
    int tempo = 500000;
    uint64_t previous = 0;
    double seconds = 0;
    for (const auto& m : messages) {
        seconds += double(m.tick - previous) * (tempo * 1e-6 / division);
        previous = m.tick;
        if (m.status == 0xff) {
            tempo = m.a;
            continue;
        }
        const int kind = m.status >> 4;
        if (kind != 8 && kind != 9)
            continue;
        if (seconds * rate >= std::numeric_limits<int>::max() / 2)
            throw std::runtime_error("MIDI exceeds maximum render duration");
        const int frame = static_cast<int>(std::nearbyint(seconds * rate));
        const size_t key = size_t((m.status & 15) * 128 + m.a);
        if (kind == 9 && m.b) {
            const int index = int(pending.size());
            if (head[key]) pending[size_t(tail[key])].next = index;
            else head[key] = index;
            tail[key] = index;
            pending.push_back({frame, 0});
        } else if (head[key]) {
            const Pending note = pending[size_t(head[key])];
            midi.onsets.push_back(note.start);
            head[key] = note.next;
            midi.bodyFrames = std::max(midi.bodyFrames, frame);
        }
    }
    std::sort(midi.onsets.begin(), midi.onsets.end());
    midi.onsets.erase(std::unique(midi.onsets.begin(), midi.onsets.end()), midi.onsets.end());
}

Midi parse(std::string_view data, int rate, TailPolicy tail, bool measure)
{
    Reader file(data);
    if (file.take(4) != "MThd")
        throw std::runtime_error("expected a Standard MIDI File");
    Reader header(file.take(file.bigEndian(4)));
    const uint32_t format = header.bigEndian(2), tracks = header.bigEndian(2), division = header.bigEndian(2);
    if (format > 1 || tracks == 0 || (format == 0 && tracks != 1) || division == 0 || division >= 32768)
        throw std::runtime_error("expected format 0/1 MIDI with PPQ timing");
    std::vector<Message> messages;
    for (uint32_t t = 0; t < tracks; ++t) {
        if (file.take(4) != "MTrk")
            throw std::runtime_error("missing MIDI track chunk");
        readTrack(Reader(file.take(file.bigEndian(4))), messages);
    }
    std::stable_sort(messages.begin(), messages.end(),
                     [](const Message& x, const Message& y) { return x.tick < y.tick; });
    Midi midi;
    if (measure)
        measureBody(messages, rate, int(division), midi);
    if (tail == TailPolicy::natural)
        prepareNatural(messages);
    if (tail == TailPolicy::custom) {
        const auto last = std::find_if(messages.rbegin(), messages.rend(), [](const Message& m) {
            const int kind = m.status >> 4;
            return kind == 8 || kind == 9 || kind == 0xb || kind == 0xe;
        });
        if (last != messages.rend()) {
            const uint64_t tick = last->tick;
            const int channel = last->status & 15;
            messages.erase(last.base(), messages.end());
            messages.push_back({tick, 0xb0 | channel, 64, 0});
            messages.push_back({tick, 0, 0, 0});
        }
    }
    uint64_t previous = 0;
    double frames = 0;
    const double scale = rate / (1000000.0 * division);
    int tempo = 500000, channel = -1;
    for (const auto& m : messages) {
        frames += double(m.tick - previous) * tempo * scale;
        previous = m.tick;
        if (frames >= std::numeric_limits<int>::max() / 2)
            throw std::runtime_error("MIDI exceeds maximum render duration");
        const int frame = static_cast<int>(tail == TailPolicy::natural ? std::nearbyint(frames)
                                                                       : std::floor(frames + 1e-7));
        if (m.status == 0xff) {
            tempo = m.a;
            continue;
        }
        if (!m.status) {
            midi.end = frame;
            continue;
        }
        const int kind = m.status >> 4, current = m.status & 15;
        if (channel < 0)
            channel = current;
        if (channel != current)
            throw std::runtime_error("multiple MIDI channels in one render job");
        switch (kind) {
        case 8:
        case 9:
            midi.events.push_back({frame, kind == 9 && m.b ? EventKind::on : EventKind::off, m.a, m.b});
            break;
        case 0xb:
            midi.events.push_back({frame, EventKind::control, m.a, m.b});
            break;
        case 0xc:
            break;                       // the job's SFZ selects the preset
        case 0xe:
            midi.events.push_back({frame, EventKind::bend, (m.a | (m.b << 7)) - 8192, 0});
            break;
        default:
            throw std::runtime_error("unsupported MIDI channel message type " + std::to_string(kind));
        }
    }
    return midi;
}

} // namespace

Midi loadMidi(const std::string& path, int rate, TailPolicy tail, bool measure)
{
    std::ifstream file(path, std::ios::binary);
    if (!file)
        throw std::runtime_error("cannot open MIDI " + path);
    const std::string data{std::istreambuf_iterator<char>(file), {}};
    try {
        return parse(data, rate, tail, measure);
    } catch (const std::exception& error) {
        throw std::runtime_error(path + ": " + error.what());
    }
}

} // namespace csh
