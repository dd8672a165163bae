// Test infrastructure for the oracle, shared by the host driver (ref_driver.cpp)
// and the GPU driver (ref_gpu.cu): the reference's batch index restated over
// cs_plan views, and the reference's sinc table.  Include after the reference's
// render_types.h and include/claysampler_b200.h.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <numeric>
#include <vector>

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

namespace refsinc {

// Renderer::Impl's sinc table (src/cuda/renderer.cpp:347-376): Kaiser beta 8.5,
// 48 taps x 2049 phases, tap-major, built in double and stored as float.
inline std::vector<float> referenceSincTable()
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

} // namespace refsinc
