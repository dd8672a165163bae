// Test infrastructure for the oracle: a C ABI over the reference's own code,
// compiled from its sources in place (see oracle/ref/Makefile).
//
//  * ref_session_plan: the reference planner (src/sfz, src/io/midi.cpp,
//    src/render/plan.cpp) run exactly as src/main.cpp:298-361 runs it, returning
//    the RenderPlan as a cs_plan image (claysampler_b200/csrc/plan_blob.hpp).
//  * ref_synthesize: the reference's per-voice render math (src/cuda/render.cu,
//    compiled as host C++) over a batch, producing the float2 (natural) or short2
//    (orig) mix the GPU finishing stages consume.
//
// Only tests and the CPU-baseline leg of bench.py load this library.
#include "render/plan.h"
#include "io/audio.h"
#include "io/midi.h"
#include "sfz/instrument.h"

#include "../../include/claysampler_b200.h"
#include "../../claysampler_b200/csrc/plan_blob.hpp"
#include "cuda_host_compat.h"

#include <climits>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

thread_local HostDim3 threadIdx, blockIdx, blockDim;

static_assert(sizeof(VoiceSpan) == sizeof(cs_voice_span), "VoiceSpan layout");
static_assert(offsetof(VoiceSpan, filteredOffset) == offsetof(cs_voice_span, filteredOffset), "VoiceSpan layout");
static_assert(offsetof(VoiceSpan, filters) == offsetof(cs_voice_span, filters), "VoiceSpan layout");
static_assert(offsetof(VoiceSpan, extraEnvelope) == offsetof(cs_voice_span, extraEnvelope), "VoiceSpan layout");
static_assert(offsetof(VoiceSpan, stereoPosition) == offsetof(cs_voice_span, stereoPosition), "VoiceSpan layout");
static_assert(sizeof(VoiceModulation) == sizeof(cs_voice_modulation), "VoiceModulation layout");
static_assert(sizeof(ControlPoint) == sizeof(cs_control_point), "ControlPoint layout");
static_assert(sizeof(TailResult) == sizeof(cs_tail_result), "TailResult layout");
static_assert(offsetof(TailResult, audio) == offsetof(cs_tail_result, audio), "TailResult layout");
static_assert(sizeof(AudioConfig) == sizeof(cs_audio_config), "AudioConfig layout");

// BatchIndex::append (src/cuda/renderer.cpp:390-460), restated for the host driver.
struct HostBatch {
    int tileFrames = 256;
    std::vector<VoiceSpan> voices;
    std::vector<Tile> tiles;
    std::vector<int> indices;
    std::vector<ControlPoint> controls;
    std::vector<VoiceModulation> modulation;
    std::vector<FilterTile> filterTiles;
    std::vector<int> filterHeads, pitchHeads, jobFrames;
    size_t frames = 0, filteredSamples = 0, pitchFrames = 0;

    void append(const cs_plan& plan)
    {
        const int count = (plan.frames + tileFrames - 1) / tileFrames;
        std::vector<int> offsets(size_t(count) + 1);
        const auto* spans = reinterpret_cast<const VoiceSpan*>(plan.spans);
        for (int s = 0; s < plan.span_count; ++s) {
            ++offsets[spans[s].begin / tileFrames];
            --offsets[(spans[s].end - 1) / tileFrames + 1];
        }
        std::partial_sum(offsets.begin(), offsets.end(), offsets.begin());
        std::vector<int> controlOffsets(size_t(plan.track_count) + 1);
        controlOffsets[0] = int(controls.size());
        for (int i = 0; i < plan.track_count; ++i) {
            const auto* first = reinterpret_cast<const ControlPoint*>(plan.points + plan.track_offsets[i]);
            const auto* last = reinterpret_cast<const ControlPoint*>(plan.points + plan.track_offsets[i + 1]);
            controls.insert(controls.end(), first, last);
            controlOffsets[size_t(i) + 1] = int(controls.size());
        }
        const int modulationOffset = int(modulation.size());
        for (int m = 0; m < plan.modulation_count; ++m) {
            auto binding = reinterpret_cast<const VoiceModulation*>(plan.modulation)[m];
            if (binding.first >= 0) {
                binding.last = controlOffsets[size_t(binding.first) + 1];
                binding.first = controlOffsets[size_t(binding.first)];
            }
            if (binding.shapeFirst >= 0) {
                binding.shapeLast = controlOffsets[size_t(binding.shapeFirst) + 1];
                binding.shapeFirst = controlOffsets[size_t(binding.shapeFirst)];
            }
            modulation.push_back(binding);
        }
        int indexCount = int(indices.size());
        for (int t = 0; t < count; ++t) {
            const int frame = t * tileFrames;
            Tile tile{frames + frame, frame, std::min(tileFrames, plan.frames - frame), indexCount, offsets[t], {}};
            std::copy_n(controlOffsets.begin(), 4, tile.controls);
            tiles.push_back(tile);
            indexCount += offsets[t];
            offsets[t] = tile.first;
        }
        indices.resize(size_t(indexCount));
        std::vector<int> tails(size_t(plan.filter_tracks), -1);
        for (int s = 0; s < plan.span_count; ++s) {
            auto voice = spans[s];
            const int index = int(voices.size());
            for (int t = voice.begin / tileFrames; t <= (voice.end - 1) / tileFrames; ++t)
                indices[size_t(offsets[t]++)] = index;
            voice.firstModulation += modulationOffset;
            if (voice.filterTrack >= 0) {
                auto& tail = tails[size_t(voice.filterTrack)];
                if (tail < 0) {
                    if (voice.variablePitch)
                        pitchHeads.push_back(index);
                    bool any = false;
                    for (const auto& filter : voice.filters)
                        any |= filter.type != FilterType::none;
                    if (any)
                        filterHeads.push_back(index);
                } else {
                    voices[size_t(tail)].nextFilteredSpan = index;
                }
                tail = index;
                voice.nextFilteredSpan = -1;
                voice.filteredOffset = filteredSamples;
                filteredSamples += size_t(voice.end - voice.begin) * voice.channels;
                if (voice.variablePitch) {
                    voice.phaseOffset = pitchFrames;
                    pitchFrames += size_t(voice.end - voice.begin);
                }
                std::copy_n(controlOffsets.begin(), 4, voice.filterControls);
                for (int frame = voice.begin; frame < voice.end; frame += tileFrames)
                    filterTiles.push_back({index, frame});
            }
            voices.push_back(voice);
        }
        frames += size_t(plan.frames);
        jobFrames.push_back(plan.frames);
    }
};

namespace ref_f32 {
#define CLAY_FLOAT_OUTPUT 1
#define renderFilterSources f32_renderFilterSources
#define prepareVoicePitch f32_prepareVoicePitch
#define applyVoiceFilters f32_applyVoiceFilters
#define renderTiles f32_renderTiles
#define scheduledTiles f32_scheduledTiles
#define scheduledSources f32_scheduledSources
#define scheduledPitch f32_scheduledPitch
#define scheduledFilters f32_scheduledFilters
#include "cuda/render.cu"
#include "ref_synth.inc"
#undef CLAY_FLOAT_OUTPUT
#undef renderFilterSources
#undef prepareVoicePitch
#undef applyVoiceFilters
#undef renderTiles
#undef scheduledTiles
#undef scheduledSources
#undef scheduledPitch
#undef scheduledFilters
} // namespace ref_f32

namespace ref_i16 {
#define CLAY_FLOAT_OUTPUT 0
#define renderFilterSources i16_renderFilterSources
#define prepareVoicePitch i16_prepareVoicePitch
#define applyVoiceFilters i16_applyVoiceFilters
#define renderTiles i16_renderTiles
#define scheduledTiles i16_scheduledTiles
#define scheduledSources i16_scheduledSources
#define scheduledPitch i16_scheduledPitch
#define scheduledFilters i16_scheduledFilters
#include "cuda/render.cu"
#include "ref_synth.inc"
} // namespace ref_i16

namespace {

// Renderer::Impl's sinc table (src/cuda/renderer.cpp:347-376): Kaiser beta 8.5,
// 48 taps x 2049 phases, tap-major, built in double and stored as float.
std::vector<float> referenceSincTable()
{
    constexpr int phases = 2048, taps = 48;
    constexpr double beta = 8.5, pi = 3.14159265358979323846;
    const auto bessel = [](double value) {
        double sum = 1, term = 1;
        for (int i = 1; i < 30; ++i) {
            term *= value * value / (4 * i * i);
            sum += term;
            if (term < 1e-14)
                break;
        }
        return sum;
    };
    const double normalization = bessel(beta);
    std::vector<float> table(size_t(taps) * (phases + 1));
    for (int tap = 0; tap < taps; ++tap) {
        for (int phase = 0; phase <= phases; ++phase) {
            const double x = tap - 23 - double(phase) / phases;
            const double f = x / 24;
            const double window = bessel(beta * std::sqrt(1 - f * f)) / normalization;
            table[size_t(tap) * (phases + 1) + phase] =
                static_cast<float>(window * (x == 0 ? 1 : std::sin(pi * x) / (pi * x)));
        }
    }
    return table;
}

struct Session {
    explicit Session(const char* library) : bank(library) {}
    clay::AudioBank bank;
    std::map<std::string, clay::Instrument> instruments;
};

void setError(char* error, size_t size, const std::string& message)
{
    if (error && size) {
        std::strncpy(error, message.c_str(), size - 1);
        error[size - 1] = 0;
    }
}

} // namespace

extern "C" {

void* ref_session_create(const char* sndfile, char* error, size_t error_size)
{
    try {
        return new Session(sndfile);
    } catch (const std::exception& e) {
        setError(error, error_size, e.what());
        return nullptr;
    }
}

void ref_session_destroy(void* session) { delete static_cast<Session*>(session); }

void ref_free(void* pointer) { std::free(pointer); }

// Plans one job as planBatch does (src/main.cpp:298-361).  tail: 0 natural,
// 1 orig, 2 custom.  Negative max_audio / tail_max mean "not given".
int ref_session_plan(void* handle, const char* sfz, const char* midiPath, int rate, int tail,
                     double maxAudio, double tailMax, int tailFadeMs, int quality, int groupVolume,
                     unsigned long long group, unsigned char** blob, size_t* size, char* error, size_t errorSize)
{
    auto& session = *static_cast<Session*>(handle);
    try {
        const auto policy = tail == 0 ? clay::TailPolicy::natural : tail == 1 ? clay::TailPolicy::orig
                                                                           : clay::TailPolicy::custom;
        auto instrument = session.instruments.find(sfz);
        if (instrument == session.instruments.end())
            instrument = session.instruments.emplace(sfz, clay::loadInstrument(sfz, session.bank)).first;
        const auto midi = clay::loadMidi(midiPath, rate, policy, groupVolume || quality);
        const int musicEnd = midi.end + 1;
        int limit = INT_MAX;
        if (policy == clay::TailPolicy::natural) {
            limit = musicEnd + naturalTailLimitSeconds * rate;
            if (maxAudio >= 0)
                limit = std::min(limit, static_cast<int>(std::floor(maxAudio * rate)));
            if (limit < musicEnd)
                throw std::runtime_error("natural render exceeds the audio duration limit");
        } else if (tailMax >= 0) {
            limit = musicEnd + static_cast<int>(std::floor(tailMax * rate));
        }
        const int customFade = static_cast<int>(std::lround((tailFadeMs >= 0 ? tailFadeMs : 100) * (rate / 1000.)));
        auto plan = clay::planRender(instrument->second, session.bank, midi, rate, 1, limit, policy);
        plan.musicEnd = musicEnd;
        plan.limit = limit;
        if (policy == clay::TailPolicy::custom && plan.tailClipped && plan.frames == limit)
            plan.fadeFrames = std::min(customFade, std::max(0, plan.frames - musicEnd));
        plan.volumeGroup = group;
        plan.bodyFrames = midi.bodyFrames;
        if (quality)
            plan.onsets = midi.onsets;

        std::vector<ControlPoint> points;
        std::vector<int64_t> offsets{0};
        for (const auto& track : plan.controls) {
            points.insert(points.end(), track.begin(), track.end());
            offsets.push_back(int64_t(points.size()));
        }
        cs_plan view{};
        view.spans = reinterpret_cast<const cs_voice_span*>(plan.spans.data());
        view.points = reinterpret_cast<const cs_control_point*>(points.data());
        view.track_offsets = offsets.data();
        view.modulation = reinterpret_cast<const cs_voice_modulation*>(plan.modulation.data());
        view.onsets = plan.onsets.data();
        view.span_count = int(plan.spans.size());
        view.track_count = int(plan.controls.size());
        view.modulation_count = int(plan.modulation.size());
        view.onset_count = int(plan.onsets.size());
        view.filter_tracks = plan.filterTracks;
        view.frames = plan.frames;
        view.music_end = plan.musicEnd;
        view.limit = plan.limit;
        view.fade_frames = plan.fadeFrames;
        view.tail_clipped = plan.tailClipped;
        view.body_frames = plan.bodyFrames;
        view.volume_group = plan.volumeGroup;
        const auto image = cs::writePlanBlob(view);
        *blob = static_cast<unsigned char*>(std::malloc(image.size()));
        std::memcpy(*blob, image.data(), image.size());
        *size = image.size();
        return 0;
    } catch (const std::exception& e) {
        setError(error, errorSize, e.what());
        return 1;
    }
}

// The session's decoded float bank (AudioBank::pcm, src/io/audio.h:32).
void ref_session_bank(void* handle, const float** pcm, size_t* floats)
{
    auto& session = *static_cast<Session*>(handle);
    *pcm = session.bank.pcm.data();
    *floats = session.bank.pcm.size();
}

void ref_sinc_table(float* out)
{
    const auto table = referenceSincTable();
    std::memcpy(out, table.data(), table.size() * sizeof(float));
}

// Mix of a batch of plans: float2 per frame (natural) or short2 (orig/custom),
// jobs concatenated in plan order.  `mix` must hold sum(frames) frames.
int ref_synthesize(const cs_plan* plans, int count, const float* bank, int natural, int threads, void* mix)
{
    static const std::vector<float> sinc = referenceSincTable();
    HostBatch batch;
    for (int i = 0; i < count; ++i)
        batch.append(plans[i]);
    if (natural)
        ref_f32::synthesize(batch, bank, sinc.data(), mix, threads);
    else
        ref_i16::synthesize(batch, bank, sinc.data(), mix, threads);
    return 0;
}

} // extern "C"
