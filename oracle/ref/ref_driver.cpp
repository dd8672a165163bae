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

#include "ref_batch.hpp"

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

using refsinc::referenceSincTable;

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
