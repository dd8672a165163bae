// Standard MIDI Files -> timed events of one render job.
//
// Reading is a pipeline over one flat list of channel and meta messages: decode
// every track (running status, tempo and end-of-track metas), merge the tracks in
// tick order, optionally measure the performance for the quality gate (note
// onsets, the end of the last note), shape the list for the tail policy (natural:
// end at the last note or the pedal release that follows it and drop what cannot
// sound; custom: end with the last channel message), then convert ticks to frames
// through the tempo map.  The rules (which messages a natural render keeps, the
// order of simultaneous messages, the frame rounding of each policy) are those of
// the reference's reader (src/io/midi.cpp), whose plans must be reproduced bit
// for bit.
#include "model.hpp"

#include <cmath>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <limits>
#include <stdexcept>
#include <string_view>

namespace clayhost {
namespace {

[[noreturn]] void fail(const std::string& message) { throw std::runtime_error(message); }

// A forward reader over bytes with the SMF integer encodings.
class Cursor {
public:
    explicit Cursor(std::string_view bytes) : rest_(bytes) {}
    bool done() const { return rest_.empty(); }

    std::string_view take(size_t count)
    {
        if (count > rest_.size())
            fail("truncated MIDI");
        const std::string_view out = rest_.substr(0, count);
        rest_.remove_prefix(count);
        return out;
    }
    int u8() { return static_cast<unsigned char>(take(1)[0]); }
    uint32_t bigEndian(int bytes)
    {
        uint32_t v = 0;
        for (int i = 0; i < bytes; ++i)
            v = v << 8 | uint32_t(u8());
        return v;
    }
    uint32_t varLength()
    {
        uint32_t v = 0;
        for (int i = 0; i < 4; ++i) {
            const int b = u8();
            v = v << 7 | uint32_t(b & 0x7f);
            if (!(b & 0x80))
                return v;
        }
        fail("invalid MIDI variable-length value");
    }

private:
    std::string_view rest_;
};

// A decoded message: status 0x80-0xef (channel), 0xff (tempo, in data1) or 0
// (end of track).
struct Msg {
    uint64_t tick;
    int status, data1, data2;
    int kind() const { return status >> 4; }
    int channel() const { return status & 15; }
    bool isNote() const { return kind() == 8 || kind() == 9; }
    bool isNoteOn() const { return kind() == 9 && data2 != 0; }
};

constexpr int kTempoMeta = 0x51, kEndMeta = 0x2f;

void decodeTrack(Cursor track, std::vector<Msg>& out)
{
    uint64_t tick = 0;
    int running = 0;
    while (!track.done()) {
        tick += track.varLength();
        int status = track.u8();
        int first = -1;
        if (status < 0x80) {                    // running status: this byte is data
            first = status;
            status = running;
            if (!status)
                fail("MIDI running status has no channel message");
        }
        if (status == 0xff) {
            const int type = track.u8();
            Cursor meta(track.take(track.varLength()));
            if (type == kTempoMeta) {
                const uint32_t tempo = meta.bigEndian(3);
                if (!tempo || !meta.done())
                    fail("invalid MIDI tempo");
                out.push_back({tick, 0xff, int(tempo), 0});
            } else if (type == kEndMeta) {
                if (!meta.done())
                    fail("invalid MIDI end-of-track");
                out.push_back({tick, 0, 0, 0});
                return;
            }
            running = 0;
            continue;
        }
        if (status >= 0xf0)
            fail("unsupported MIDI system or SysEx message");
        running = status;
        if (first < 0)
            first = track.u8();
        const int kind = status >> 4;
        const int second = kind == 0xc || kind == 0xd ? 0 : track.u8();
        if (first >= 0x80 || second >= 0x80)
            fail("invalid MIDI data byte");
        out.push_back({tick, status, first, second});
    }
    fail("missing MIDI end-of-track");
}

// Onsets and the end of the last note, with note-offs matched first-in first-out
// per channel and key, in seconds through the tempo map rounded to frames.
void measure(const std::vector<Msg>& msgs, int rate, int division, Score& score)
{
    std::vector<std::vector<int>> open(16 * 128);     // pending onset frames per channel and key
    std::vector<size_t> head(16 * 128, 0);
    int tempo = 500000;
    uint64_t lastTick = 0;
    double seconds = 0;
    for (const Msg& m : msgs) {
        seconds += double(m.tick - lastTick) * (tempo * 1e-6 / division);
        lastTick = m.tick;
        if (m.status == 0xff) {
            tempo = m.data1;
            continue;
        }
        if (!m.isNote())
            continue;
        if (seconds * rate >= std::numeric_limits<int>::max() / 2)
            fail("MIDI exceeds maximum render duration");
        const int frame = static_cast<int>(std::nearbyint(seconds * rate));
        const size_t slot = size_t(m.channel()) * 128 + size_t(m.data1);
        if (m.isNoteOn()) {
            open[slot].push_back(frame);
        } else if (head[slot] < open[slot].size()) {
            score.onsets.push_back(open[slot][head[slot]++]);
            score.bodyFrames = std::max(score.bodyFrames, frame);
        }
    }
    std::sort(score.onsets.begin(), score.onsets.end());
    score.onsets.erase(std::unique(score.onsets.begin(), score.onsets.end()), score.onsets.end());
}

// Order of simultaneous messages in a natural render: controllers and other
// channel messages, then note-offs, then note-ons.
int simultaneousRank(const Msg& m)
{
    if (m.isNoteOn())
        return 2;
    return m.isNote() ? 1 : 0;
}

// Natural tail: the render ends at the last note-off, or later at the first
// release of a pedal (sustain, sostenuto, hold) that was down at that point; what
// follows is dropped, as are program changes, bank select, volume / pan / effect
// sends, and all-notes-off / all-sound-off before the last note.  Volume 100 and
// centred pan are set at the start, and the pedals are released at the end.
void shapeNatural(std::vector<Msg>& msgs)
{
    std::vector<int> held(16 * 128, 0);
    uint64_t lastNoteOff = 0;
    int channel = -1;
    for (const Msg& m : msgs) {
        if (!m.isNote())
            continue;
        int& count = held[size_t(m.channel()) * 128 + size_t(m.data1)];
        if (m.isNoteOn()) {
            ++count;
        } else if (count > 0) {
            --count;
            if (channel >= 0 && channel != m.channel())
                fail("multiple MIDI channels in one render job");
            channel = m.channel();
            lastNoteOff = m.tick;
        }
    }
    if (channel < 0)
        fail("natural rendering requires a complete MIDI note");
    static constexpr int kPedals[] = {64, 66, 69};
    bool down[3] = {false, false, false};
    uint64_t end = lastNoteOff;
    for (const Msg& m : msgs) {
        if (m.kind() != 0xb)
            continue;
        for (int p = 0; p < 3; ++p) {
            if (m.data1 != kPedals[p])
                continue;
            if (m.tick <= end)
                down[p] = m.data2 >= 64;
            else if (down[p] && m.data2 < 64) {
                end = m.tick;
                down[p] = false;
            }
        }
    }
    const auto dropped = [&](const Msg& m) {
        if (!m.status || m.tick > end || m.kind() == 0xc)
            return true;
        if (m.kind() != 0xb)
            return false;
        switch (m.data1) {
        case 0: case 7: case 10: case 32: case 91: case 93: return true;
        case 120: case 123: return m.tick >= lastNoteOff;
        default: return false;
        }
    };
    msgs.erase(std::remove_if(msgs.begin(), msgs.end(), dropped), msgs.end());
    const int control = 0xb0 | channel;
    msgs.insert(msgs.begin(), {{0, control, 7, 100}, {0, control, 10, 64}});
    std::stable_sort(msgs.begin(), msgs.end(), [](const Msg& a, const Msg& b) {
        return a.tick != b.tick ? a.tick < b.tick : simultaneousRank(a) < simultaneousRank(b);
    });
    for (const int cc : kPedals)
        msgs.push_back({end, control, cc, 0});
    msgs.push_back({end, 0, 0, 0});
}

// Custom tail: the render ends with the last note, controller or bend message; the
// sustain pedal is released there.
void shapeCustom(std::vector<Msg>& msgs)
{
    const auto last = std::find_if(msgs.rbegin(), msgs.rend(), [](const Msg& m) {
        return m.isNote() || m.kind() == 0xb || m.kind() == 0xe;
    });
    if (last == msgs.rend())
        return;
    const uint64_t tick = last->tick;
    const int channel = last->channel();
    msgs.erase(last.base(), msgs.end());
    msgs.push_back({tick, 0xb0 | channel, 64, 0});
    msgs.push_back({tick, 0, 0, 0});
}

Score decode(std::string_view data, int rate, TailPolicy tail, bool measured)
{
    Cursor file(data);
    if (file.take(4) != "MThd")
        fail("expected a Standard MIDI File");
    Cursor header(file.take(file.bigEndian(4)));
    const uint32_t format = header.bigEndian(2), tracks = header.bigEndian(2), division = header.bigEndian(2);
    if (format > 1 || tracks == 0 || (format == 0 && tracks != 1) || division == 0 || division >= 32768)
        fail("expected format 0/1 MIDI with PPQ timing");
    std::vector<Msg> msgs;
    for (uint32_t t = 0; t < tracks; ++t) {
        if (file.take(4) != "MTrk")
            fail("missing MIDI track chunk");
        decodeTrack(Cursor(file.take(file.bigEndian(4))), msgs);
    }
    std::stable_sort(msgs.begin(), msgs.end(), [](const Msg& a, const Msg& b) { return a.tick < b.tick; });
    Score score;
    if (measured)
        measure(msgs, rate, int(division), score);
    if (tail == TailPolicy::natural)
        shapeNatural(msgs);
    else if (tail == TailPolicy::custom)
        shapeCustom(msgs);
    // Ticks to frames: natural renders round to the nearest frame, the others
    // take the frame the tick falls in.
    const double scale = rate / (1000000.0 * division);
    int tempo = 500000;
    uint64_t lastTick = 0;
    double frames = 0;
    int channel = -1;
    for (const Msg& m : msgs) {
        frames += double(m.tick - lastTick) * tempo * scale;
        lastTick = m.tick;
        if (frames >= std::numeric_limits<int>::max() / 2)
            fail("MIDI exceeds maximum render duration");
        const int frame = static_cast<int>(tail == TailPolicy::natural ? std::nearbyint(frames) : std::floor(frames + 1e-7));
        if (m.status == 0xff) {
            tempo = m.data1;
            continue;
        }
        if (!m.status) {
            score.endFrame = frame;
            continue;
        }
        if (channel < 0)
            channel = m.channel();
        if (channel != m.channel())
            fail("multiple MIDI channels in one render job");
        switch (m.kind()) {
        case 0x8:
        case 0x9:
            score.events.push_back({frame, m.isNoteOn() ? EventType::noteOn : EventType::noteOff, m.data1, m.data2});
            break;
        case 0xb:
            score.events.push_back({frame, EventType::control, m.data1, m.data2});
            break;
        case 0xc:                       // the job selects the instrument, as sfizz_render does
            break;
        case 0xe:
            score.events.push_back({frame, EventType::bend, (m.data1 | (m.data2 << 7)) - 8192, 0});
            break;
        default:
            fail("unsupported MIDI channel message type " + std::to_string(m.kind()));
        }
    }
    return score;
}

} // namespace

Score readScore(const std::string& path, int rate, TailPolicy tail, bool measured)
{
    std::ifstream in(std::filesystem::u8path(path), std::ios::binary);
    if (!in)
        fail("cannot open MIDI " + path);
    const std::string data{std::istreambuf_iterator<char>(in), {}};
    try {
        return decode(data, rate, tail, measured);
    } catch (const std::exception& error) {
        fail(path + ": " + error.what());
    }
}

} // namespace clayhost
