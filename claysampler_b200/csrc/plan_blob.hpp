// Flat byte image of one cs_plan, used to move planned jobs between processes and
// into Python (numpy views) without re-planning.  Layout, all little-endian:
//
//   "CSPL" u32 version=1
//   i32 filter_tracks frames music_end limit fade_frames tail_clipped body_frames
//   i32 span_count track_count modulation_count onset_count reserved
//   u64 volume_group point_count
//   cs_voice_span[span_count] | i64 track_offsets[track_count+1]
//   cs_control_point[point_count] | cs_voice_modulation[modulation_count] | i32 onsets[onset_count]
#pragma once

#include "../../include/claysampler_b200.h"

#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace cs {

constexpr size_t planBlobHeader = 72;

static_assert(sizeof(cs_voice_span) == 472, "cs_voice_span must match the reference VoiceSpan");
static_assert(sizeof(cs_control_point) == 12, "cs_control_point must match ControlPoint");
static_assert(sizeof(cs_voice_modulation) == 24, "cs_voice_modulation must match VoiceModulation");
static_assert(sizeof(cs_tail_result) == 112, "cs_tail_result must match TailResult");
static_assert(sizeof(cs_audio_config) == 72, "cs_audio_config must match AudioConfig");

inline std::vector<unsigned char> writePlanBlob(const cs_plan& plan)
{
    const int64_t points = plan.track_count ? plan.track_offsets[plan.track_count] : 0;
    const size_t bytes = planBlobHeader + size_t(plan.span_count) * sizeof(cs_voice_span) +
        size_t(plan.track_count + 1) * sizeof(int64_t) + size_t(points) * sizeof(cs_control_point) +
        size_t(plan.modulation_count) * sizeof(cs_voice_modulation) + size_t(plan.onset_count) * sizeof(int32_t);
    std::vector<unsigned char> out(bytes);
    unsigned char* p = out.data();
    const auto put = [&](const void* data, size_t size) {
        if (size) std::memcpy(p, data, size);
        p += size;
    };
    const uint32_t version = 1;
    put("CSPL", 4);
    put(&version, 4);
    const int32_t fields[12] = {plan.filter_tracks, plan.frames, plan.music_end, plan.limit, plan.fade_frames,
        plan.tail_clipped, plan.body_frames, plan.span_count, plan.track_count, plan.modulation_count,
        plan.onset_count, 0};
    put(fields, sizeof fields);
    const uint64_t tail[2] = {plan.volume_group, uint64_t(points)};
    put(tail, sizeof tail);
    // Spans are written with their one padding gap (after nextFilteredSpan) zeroed,
    // so equal plans have equal images.
    constexpr size_t gap = offsetof(cs_voice_span, nextFilteredSpan) + sizeof(int32_t);
    static_assert(offsetof(cs_voice_span, filteredOffset) - gap == 4, "cs_voice_span padding");
    for (int s = 0; s < plan.span_count; ++s) {
        unsigned char* at = p;
        put(&plan.spans[s], sizeof(cs_voice_span));
        std::memset(at + gap, 0, 4);
    }
    if (plan.track_count) {
        put(plan.track_offsets, size_t(plan.track_count + 1) * sizeof(int64_t));
    } else {
        const int64_t zero = 0;
        put(&zero, sizeof zero);
    }
    put(plan.points, size_t(points) * sizeof(cs_control_point));
    put(plan.modulation, size_t(plan.modulation_count) * sizeof(cs_voice_modulation));
    put(plan.onsets, size_t(plan.onset_count) * sizeof(int32_t));
    return out;
}

// Returns a view whose arrays point into `blob` (which must outlive it).
inline cs_plan readPlanBlob(const unsigned char* blob, size_t size)
{
    if (size < planBlobHeader || std::memcmp(blob, "CSPL", 4))
        throw std::runtime_error("not a plan image");
    int32_t fields[12];
    uint64_t tail[2];
    std::memcpy(fields, blob + 8, sizeof fields);
    std::memcpy(tail, blob + 56, sizeof tail);
    cs_plan plan{};
    plan.filter_tracks = fields[0];
    plan.frames = fields[1];
    plan.music_end = fields[2];
    plan.limit = fields[3];
    plan.fade_frames = fields[4];
    plan.tail_clipped = fields[5];
    plan.body_frames = fields[6];
    plan.span_count = fields[7];
    plan.track_count = fields[8];
    plan.modulation_count = fields[9];
    plan.onset_count = fields[10];
    plan.volume_group = tail[0];
    size_t offset = planBlobHeader;
    plan.spans = reinterpret_cast<const cs_voice_span*>(blob + offset);
    offset += size_t(plan.span_count) * sizeof(cs_voice_span);
    plan.track_offsets = reinterpret_cast<const int64_t*>(blob + offset);
    offset += size_t(plan.track_count + 1) * sizeof(int64_t);
    plan.points = reinterpret_cast<const cs_control_point*>(blob + offset);
    offset += size_t(tail[1]) * sizeof(cs_control_point);
    plan.modulation = reinterpret_cast<const cs_voice_modulation*>(blob + offset);
    offset += size_t(plan.modulation_count) * sizeof(cs_voice_modulation);
    plan.onsets = reinterpret_cast<const int32_t*>(blob + offset);
    offset += size_t(plan.onset_count) * sizeof(int32_t);
    if (offset != size)
        throw std::runtime_error("truncated plan image");
    return plan;
}

} // namespace cs
