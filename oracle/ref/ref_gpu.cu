// Test infrastructure for the oracle: the reference's own render kernels
// (src/cuda/render.cu, compiled here by nvcc from the reference's sources in
// place, with the reference's NVRTC defaults: FMA contraction on, float output)
// launched on the GPU over the same batch index the host driver builds
// (ref_batch.hpp), in the reference's launch order and shapes
// (src/cuda/renderer.cpp:1047-1107, 693-717): variable-pitch phases, filter
// sources, filter chains, then the mix tiles, one segment covering every frame.
//
// This is the float bus of "the reference's own render on the same GPU".  Only
// tests load this library (oracle/_ref/libclayref_gpu.so); the product never does.
#define CLAY_FLOAT_OUTPUT 1
#include "render.cu"

#include "../../include/claysampler_b200.h"
#include "ref_batch.hpp"

#include <cstring>
#include <stdexcept>
#include <string>

static_assert(sizeof(VoiceSpan) == sizeof(cs_voice_span), "VoiceSpan layout");
static_assert(sizeof(ControlPoint) == sizeof(cs_control_point), "ControlPoint layout");
static_assert(sizeof(VoiceModulation) == sizeof(cs_voice_modulation), "VoiceModulation layout");

namespace {

thread_local std::string lastError;

struct DeviceBuffers {
    std::vector<void*> owned;
    ~DeviceBuffers()
    {
        for (void* p : owned)
            cudaFree(p);
    }
    template <class T>
    T* upload(const std::vector<T>& items, size_t minimum = 1)
    {
        void* p = nullptr;
        const size_t bytes = std::max(items.size(), minimum) * sizeof(T);
        check(cudaMalloc(&p, bytes), "allocation");
        owned.push_back(p);
        check(cudaMemset(p, 0, bytes), "clear");
        if (!items.empty())
            check(cudaMemcpy(p, items.data(), items.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
        return static_cast<T*>(p);
    }
    void* zeros(size_t bytes)
    {
        void* p = nullptr;
        check(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "allocation");
        owned.push_back(p);
        check(cudaMemset(p, 0, std::max<size_t>(bytes, 16)), "clear");
        return p;
    }
    static void check(cudaError_t status, const char* what)
    {
        if (status != cudaSuccess)
            throw std::runtime_error(std::string("reference GPU render: ") + what + ": " + cudaGetErrorString(status));
    }
};

} // namespace

extern "C" {

const char* ref_gpu_last_error(void) { return lastError.c_str(); }

// Float mix (float2 per frame, jobs concatenated in plan order) of `count` plans
// rendered by the reference's kernels on the current device.  `mix` is host
// memory of sum(frames) float2.  Returns 0 on success.
int ref_gpu_synthesize_timed(const cs_plan* plans, int count, const float* bank, size_t bankFloats, void* mix,
                             int repeats, float* ms);

int ref_gpu_synthesize(const cs_plan* plans, int count, const float* bank, size_t bankFloats, void* mix)
{
    return ref_gpu_synthesize_timed(plans, count, bank, bankFloats, mix, 0, nullptr);
}

// As ref_gpu_synthesize; with `repeats` > 0 the launch sequence then runs that
// many more times on the device-resident batch and `ms` receives the mean device
// time of one sequence (CUDA events around the launches).
int ref_gpu_synthesize_timed(const cs_plan* plans, int count, const float* bank, size_t bankFloats, void* mix,
                             int repeats, float* ms)
{
    try {
        HostBatch batch;
        for (int i = 0; i < count; ++i)
            batch.append(plans[i]);
        int lastFrame = 0;
        for (int frames : batch.jobFrames)
            lastFrame = std::max(lastFrame, frames);
        const int first = 0, end = lastFrame, frames = lastFrame;
        const int tileFrames = batch.tileFrames;
        DeviceBuffers d;
        const std::vector<float> sincTable = refsinc::referenceSincTable();
        std::vector<float> samples(bank, bank + bankFloats);
        const float* dSamples = d.upload(samples);
        const float* dSinc = d.upload(sincTable);
        VoiceSpan* dVoices = d.upload(batch.voices);
        const Tile* dTiles = d.upload(batch.tiles);
        const int* dIndices = d.upload(batch.indices);
        const ControlPoint* dControls = d.upload(batch.controls);
        const VoiceModulation* dModulation = d.upload(batch.modulation);
        const FilterTile* dFilterTiles = d.upload(batch.filterTiles);
        const int* dFilterHeads = d.upload(batch.filterHeads);
        const int* dPitchHeads = d.upload(batch.pitchHeads);
        auto* dFiltered = static_cast<float*>(d.zeros(batch.filteredSamples * sizeof(float)));
        auto* dPhase = static_cast<double*>(d.zeros(batch.pitchFrames * sizeof(double)));
        auto* dStates = static_cast<VoiceState*>(d.zeros(batch.voices.size() * sizeof(VoiceState)));
        auto* dOutput = static_cast<float2*>(d.zeros(batch.frames * sizeof(float2)));
        // One launch per stage, as the reference launches them for one segment; the
        // chain kernels take a thread per chain, the tile kernels a CTA per tile of
        // tileFrames threads (every kernel bounds-checks its index).
        constexpr int chainThreads = 32;
        const int pitchCount = int(batch.pitchHeads.size());
        const int sourceCount = int(batch.filterTiles.size());
        const int filterCount = int(batch.filterHeads.size());
        const int tileCount = int(batch.tiles.size());
        const auto sequence = [&] {
            if (pitchCount)
                prepareVoicePitch<<<(pitchCount + chainThreads - 1) / chainThreads, chainThreads>>>(
                    dVoices, dPitchHeads, dControls, dModulation, dPhase, dStates, first, end, frames, pitchCount);
            if (sourceCount)
                renderFilterSources<<<sourceCount, tileFrames>>>(dSamples, dSinc, dVoices, dFilterTiles, dControls,
                                                                 dModulation, dPhase, dFiltered, first, end, frames, 0);
            if (filterCount)
                applyVoiceFilters<<<(filterCount + chainThreads - 1) / chainThreads, chainThreads>>>(
                    dVoices, dFilterHeads, dControls, dModulation, dFiltered, dStates, first, end, frames, filterCount);
            if (tileCount)
                renderTiles<<<tileCount, tileFrames>>>(dSamples, dSinc, dVoices, dTiles, dIndices, dControls,
                                                       dModulation, dFiltered, dOutput, first, end, frames, 0);
        };
        sequence();
        DeviceBuffers::check(cudaGetLastError(), "launch");
        DeviceBuffers::check(cudaDeviceSynchronize(), "render");
        if (repeats > 0 && ms) {
            // Chain state restarts from zero for every run of the sequence.
            const size_t stateBytes = std::max<size_t>(batch.voices.size() * sizeof(VoiceState), 16);
            cudaEvent_t start, stop;
            DeviceBuffers::check(cudaEventCreate(&start), "event");
            DeviceBuffers::check(cudaEventCreate(&stop), "event");
            float total = 0;
            for (int k = 0; k < repeats; ++k) {
                DeviceBuffers::check(cudaMemset(dStates, 0, stateBytes), "clear");
                DeviceBuffers::check(cudaEventRecord(start), "event");
                sequence();
                DeviceBuffers::check(cudaEventRecord(stop), "event");
                DeviceBuffers::check(cudaEventSynchronize(stop), "render");
                float once = 0;
                DeviceBuffers::check(cudaEventElapsedTime(&once, start, stop), "timing");
                total += once;
            }
            cudaEventDestroy(start);
            cudaEventDestroy(stop);
            *ms = total / float(repeats);
        }
        DeviceBuffers::check(cudaMemcpy(mix, dOutput, batch.frames * sizeof(float2), cudaMemcpyDeviceToHost),
                             "download");
        return 0;
    } catch (const std::exception& e) {
        lastError = e.what();
        return 1;
    }
}

} // extern "C"
