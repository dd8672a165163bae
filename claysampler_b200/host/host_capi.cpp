// C ABI of the host library (include/claysampler_host.h).
#include "../../include/claysampler_host.h"
#include "../csrc/plan_blob.hpp"
#include "model.hpp"

#include <array>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>

#include <fcntl.h>
#include <unistd.h>

namespace {

thread_local std::string lastError;

template <class F>
int guarded(F&& body)
{
    try {
        body();
        return 0;
    } catch (const std::exception& e) {
        lastError = e.what();
        return 1;
    }
}

std::array<unsigned char, 44> waveHeader(uint32_t bytes, int rate, int channels)
{
    std::array<unsigned char, 44> header{};
    const auto put = [&](size_t offset, uint32_t value, int width) {
        for (int i = 0; i < width; ++i)
            header[offset + size_t(i)] = static_cast<unsigned char>(value >> (8 * i));
    };
    std::memcpy(header.data(), "RIFF", 4);
    put(4, bytes + 36, 4);
    std::memcpy(header.data() + 8, "WAVEfmt ", 8);
    put(16, 16, 4);
    put(20, 1, 2);
    put(22, uint32_t(channels), 2);
    put(24, uint32_t(rate), 4);
    put(28, uint32_t(rate * channels * 2), 4);
    put(32, uint32_t(channels * 2), 2);
    put(34, 16, 2);
    std::memcpy(header.data() + 36, "data", 4);
    put(40, bytes, 4);
    return header;
}

void syncPath(const std::filesystem::path& path, int flags)
{
    const int fd = ::open(path.c_str(), flags);
    if (fd < 0)
        throw std::runtime_error("cannot open for sync " + path.string());
    const int status = ::fsync(fd);
    const int closed = ::close(fd);
    if (status || closed)
        throw std::runtime_error("cannot sync " + path.string());
}

} // namespace

struct cs_host {
    clayhost::SampleBank bank;
    std::map<std::string, clayhost::Instrument> instruments;
};

extern "C" {

const char* cs_host_last_error(void) { return lastError.c_str(); }

int cs_host_create(cs_host** out)
{
    return guarded([&] {
        if (!out)
            throw std::runtime_error("null output handle");
        *out = new cs_host();
    });
}

void cs_host_destroy(cs_host* host) { delete host; }
void cs_host_free(void* pointer) { std::free(pointer); }

int cs_host_plan(cs_host* host, const char* sfz, const char* midiPath, int rate, int tail, double maxAudio,
                 double tailMax, int tailFadeMs, int quality, int groupVolume, uint64_t group, void** image,
                 size_t* size)
{
    return guarded([&] {
        if (!host || !sfz || !midiPath || !image || !size)
            throw std::runtime_error("null argument");
        const auto policy = tail == 0 ? clayhost::TailPolicy::natural : tail == 1 ? clayhost::TailPolicy::orig
                                                                                     : clayhost::TailPolicy::custom;
        auto instrument = host->instruments.find(sfz);
        if (instrument == host->instruments.end())
            instrument = host->instruments.emplace(sfz, clayhost::readInstrument(sfz, host->bank)).first;
        const clayhost::Score midi = clayhost::readScore(midiPath, rate, policy, groupVolume || quality);
        const int musicEnd = midi.endFrame + 1;
        int limit = INT_MAX;
        if (policy == clayhost::TailPolicy::natural) {
            limit = musicEnd + CS_NATURAL_TAIL_LIMIT_SECONDS * rate;
            if (maxAudio >= 0)
                limit = std::min(limit, static_cast<int>(std::floor(maxAudio * rate)));
            if (limit < musicEnd)
                throw std::runtime_error("natural render exceeds the audio duration limit");
        } else if (tailMax >= 0) {
            limit = musicEnd + static_cast<int>(std::floor(tailMax * rate));
        }
        const int customFade = static_cast<int>(std::lround((tailFadeMs >= 0 ? tailFadeMs : 100) * (rate / 1000.)));
        clayhost::Plan plan = clayhost::planJob(instrument->second, host->bank, midi, rate, 1, limit, policy);
        plan.musicEnd = musicEnd;
        plan.limit = limit;
        if (policy == clayhost::TailPolicy::custom && plan.tailClipped && plan.frames == limit)
            plan.fadeFrames = std::min(customFade, std::max(0, plan.frames - musicEnd));
        plan.volumeGroup = group;
        plan.bodyFrames = midi.bodyFrames;
        if (quality)
            plan.onsets = midi.onsets;
        std::vector<cs_control_point> points;
        std::vector<int64_t> offsets{0};
        for (const auto& track : plan.tracks) {
            points.insert(points.end(), track.begin(), track.end());
            offsets.push_back(int64_t(points.size()));
        }
        cs_plan view{};
        view.spans = plan.spans.data();
        view.points = points.data();
        view.track_offsets = offsets.data();
        view.modulation = plan.bindings.data();
        view.onsets = plan.onsets.data();
        view.span_count = int(plan.spans.size());
        view.track_count = int(plan.tracks.size());
        view.modulation_count = int(plan.bindings.size());
        view.onset_count = int(plan.onsets.size());
        view.filter_tracks = plan.filterTracks;
        view.frames = plan.frames;
        view.music_end = plan.musicEnd;
        view.limit = plan.limit;
        view.fade_frames = plan.fadeFrames;
        view.tail_clipped = plan.tailClipped;
        view.body_frames = plan.bodyFrames;
        view.volume_group = plan.volumeGroup;
        const auto bytes = cs::writePlanBlob(view);
        void* out = std::malloc(bytes.size());
        if (!out)
            throw std::runtime_error("out of host memory");
        std::memcpy(out, bytes.data(), bytes.size());
        *image = out;
        *size = bytes.size();
    });
}

int cs_host_check_sfz(const char* sfz, int* regions)
{
    return guarded([&] {
        if (!sfz || !regions)
            throw std::runtime_error("null argument");
        clayhost::SampleBank bank;
        *regions = int(clayhost::readInstrument(sfz, bank).regions.size());
    });
}

int cs_host_bank(cs_host* host, const float** pcm, size_t* floats)
{
    return guarded([&] {
        if (!host || !pcm || !floats)
            throw std::runtime_error("null argument");
        *pcm = host->bank.pcm.data();
        *floats = host->bank.pcm.size();
    });
}

int cs_host_release_bank(cs_host* host)
{
    return guarded([&] {
        if (!host)
            throw std::runtime_error("null host");
        host->bank.releaseDecoded();
    });
}

int cs_write_wave(const char* path, const int16_t* pcm, int dataFrames, int frames, int rate, int channels)
{
    return guarded([&] {
        const int stride = channels * 2;
        if (!path || frames <= 0 || dataFrames < 0 || dataFrames > frames ||
            static_cast<uint64_t>(frames) * uint64_t(stride) + 36 > UINT32_MAX)
            throw std::runtime_error("output exceeds PCM16 WAV limits");
        const std::filesystem::path destination(path);
        const auto temporary = destination.parent_path() /
            ("claysampler." + std::to_string(::getpid()) + "." + destination.filename().string() + ".part");
        {
            std::ofstream file(temporary, std::ios::binary | std::ios::trunc);
            const auto header = waveHeader(uint32_t(frames) * uint32_t(stride), rate, channels);
            file.write(reinterpret_cast<const char*>(header.data()), std::streamsize(header.size()));
            if (dataFrames)
                file.write(reinterpret_cast<const char*>(pcm), std::streamsize(size_t(dataFrames) * size_t(stride)));
            static const char zeros[16384] = {};
            for (size_t remaining = size_t(frames - dataFrames) * size_t(stride); remaining;) {
                const size_t count = std::min(remaining, sizeof zeros);
                file.write(zeros, std::streamsize(count));
                remaining -= count;
            }
            file.close();
            if (!file)
                throw std::runtime_error("cannot write WAV " + destination.string());
        }
        syncPath(temporary, O_WRONLY);
        std::filesystem::rename(temporary, destination);
        syncPath(destination.has_parent_path() ? destination.parent_path() : ".", O_RDONLY | O_DIRECTORY);
    });
}

int cs_wave_complete(const char* path, int rate, int channels)
{
    std::ifstream input(path, std::ios::binary | std::ios::ate);
    if (!input)
        return 0;
    const std::streamoff size = input.tellg();
    if (size <= 44 || size - 44 > std::streamoff(UINT32_MAX - 36) || (size - 44) % (channels * 2))
        return 0;
    std::array<unsigned char, 44> header;
    input.seekg(0);
    return input.read(reinterpret_cast<char*>(header.data()), std::streamsize(header.size())) &&
        header == waveHeader(static_cast<uint32_t>(size - 44), rate, channels);
}

} // extern "C"
