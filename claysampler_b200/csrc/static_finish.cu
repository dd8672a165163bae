// Natural-tail finishing that allocates nothing, for callers that cannot call
// cudaMalloc while they render: a real-time audio host rendering inside its
// audio callback (a device allocation can block for milliseconds or synchronise
// the device, which breaks the callback's deadline), or an application embedding
// the renderer that owns the whole device-memory budget itself.
//
// The stage's intermediates — per-block stereo power and peak, per-window mono
// stats, the mono PCM16, the per-job search reductions and the job tables — live in one file-scope device array
// of fixed size instead of the renderer's arena.  Its limit is
// CS_STATIC_FINISH_MAX_FRAMES frames and CS_STATIC_FINISH_MAX_JOBS jobs per call.
// Every call reuses the same array and leaves the last call's contents in it;
// every word a call reads is written earlier in the same call (the job tables by
// a set-up kernel from the job records, which the launch carries as its
// parameter), so nothing needs clearing.  Calls whose work overlaps on the GPU (on different streams, or from
// different threads) race on the array and must be serialised by the caller.
#include "kernels.cuh"

#include <cmath>
#include <mutex>
#include <stdexcept>
#include <string>

namespace cs {
namespace {

constexpr size_t kMaxFrames = CS_STATIC_FINISH_MAX_FRAMES;
constexpr size_t kMaxJobs = CS_STATIC_FINISH_MAX_JOBS;
constexpr size_t kMaxBlocks = kMaxFrames / kBlockFrames + kMaxJobs;
constexpr size_t kMinWindow = 400;           // smallest accepted 50 ms window (8 kHz)
constexpr size_t kMaxWindows = kMaxFrames / kMinWindow + kMaxJobs;

constexpr size_t alignUp(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kJobsAt = 0;
constexpr size_t kBlockJobAt = alignUp(kJobsAt + kMaxJobs * sizeof(JobInfo));
constexpr size_t kWindowJobAt = alignUp(kBlockJobAt + kMaxBlocks * sizeof(int));
constexpr size_t kStereoAt = alignUp(kWindowJobAt + kMaxWindows * sizeof(int));
constexpr size_t kWindowsAt = alignUp(kStereoAt + kMaxBlocks * sizeof(StereoStats));
constexpr size_t kMonoAt = alignUp(kWindowsAt + kMaxWindows * sizeof(MonoStats));
constexpr size_t kScansAt = alignUp(kMonoAt + kMaxFrames * sizeof(short));
constexpr size_t kScratchBytes = alignUp(kScansAt + kMaxJobs * sizeof(JobScan));

static __device__ __align__(256) unsigned char gFinishScratch[kScratchBytes];

std::mutex gSetup;
unsigned char* gScratchAddress[64] = {};

// Device address of the array on the current device.  In host code the array's
// name is only a host-side stand-in, so the address is looked up once per device
// (with that device current) and cached.
unsigned char* scratchOnCurrentDevice()
{
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64)
        throw std::runtime_error("no usable current CUDA device");
    std::lock_guard<std::mutex> lock(gSetup);
    if (!gScratchAddress[device]) {
        void* address = nullptr;
        const cudaError_t status = cudaGetSymbolAddress(&address, gFinishScratch);
        if (status != cudaSuccess)
            throw std::runtime_error(std::string("static finishing scratch: ") + cudaGetErrorString(status));
        gScratchAddress[device] = static_cast<unsigned char*>(address);
    }
    return gScratchAddress[device];
}

thread_local std::string lastStaticError;

// The job table travels to the device as a kernel parameter (4 KB of records
// copied into the launch itself), so the call stages nothing through pageable
// memory and reads no host memory after it returns.
struct FinishTable {
    cs_finish_job jobs[kMaxJobs];
    int count, window;
};
static_assert(sizeof(FinishTable) <= 32764, "kernel parameter limit");

// One CTA of kMaxJobs threads: thread j owns job j.  Exclusive scans of the jobs'
// frames, 1024-frame blocks and tail windows give each job's offsets; then the
// CTA writes the job of every block and window (a binary search over the scanned
// offsets in shared memory).
__global__ void __launch_bounds__(kMaxJobs) finishSetupKernel(FinishTable t, JobInfo* jobs, int* blockJob,
                                                              int* windowJob)
{
    __shared__ unsigned long long frameBase[kMaxJobs];
    __shared__ int blockBase[kMaxJobs + 1], windowBase[kMaxJobs + 1];
    const int j = int(threadIdx.x);
    const int frames = j < t.count ? t.jobs[j].frames : 0;
    const int blocks = (frames + kBlockFrames - 1) / kBlockFrames;
    const int windows = (frames + t.window - 1) / t.window;
    frameBase[j] = (unsigned long long)frames;
    blockBase[j + 1] = blocks;
    windowBase[j + 1] = windows;
    if (j == 0)
        blockBase[0] = windowBase[0] = 0;
    __syncthreads();
    // Inclusive scans (Hillis-Steele); frameBase is made exclusive afterwards.
    for (int d = 1; d < kMaxJobs; d <<= 1) {
        const unsigned long long f = j >= d ? frameBase[j - d] : 0ull;
        const int b = j >= d ? blockBase[j + 1 - d] : 0, w = j >= d ? windowBase[j + 1 - d] : 0;
        __syncthreads();
        frameBase[j] += f;
        blockBase[j + 1] += b;
        windowBase[j + 1] += w;
        __syncthreads();
    }
    if (j < t.count) {
        JobInfo info{};
        info.offset = frameBase[j] - (unsigned long long)frames;
        info.frames = frames;
        info.musicEnd = t.jobs[j].music_end;
        info.limit = t.jobs[j].limit;
        info.fade = t.jobs[j].fade_frames;
        info.blockFirst = blockBase[j];
        info.windowFirst = windowBase[j];
        jobs[j] = info;
    }
    const auto owner = [](const int* base, int count, int item) {
        int low = 0, high = count;                 // base[low] <= item < base[high]
        while (low + 1 < high) {
            const int mid = (low + high) >> 1;
            if (base[mid] <= item) low = mid;
            else high = mid;
        }
        return low;
    };
    for (int b = j; b < blockBase[t.count]; b += kMaxJobs)
        blockJob[b] = owner(blockBase, t.count, b);
    for (int w = j; w < windowBase[t.count]; w += kMaxJobs)
        windowJob[w] = owner(windowBase, t.count, w);
}

} // namespace
} // namespace cs

extern "C" int cs_finish_natural_static(const float* mix, const cs_finish_job* jobs, int count, int rate, int window,
                                        int16_t* packed, cs_tail_result* results, void* stream)
{
    using namespace cs;
    try {
        if (!mix || !jobs || !packed || !results || count <= 0)
            throw std::invalid_argument("cs_finish_natural_static: null buffer or empty job list");
        if (size_t(count) > kMaxJobs)
            throw std::invalid_argument("cs_finish_natural_static: " + std::to_string(count) + " jobs exceed the limit of " +
                                        std::to_string(kMaxJobs));
        if (rate <= 0 || window < int(kMinWindow))
            throw std::invalid_argument("cs_finish_natural_static: invalid rate or window");
        FinishTable table;
        table.count = count;
        table.window = window;
        size_t frames = 0;
        int blocks = 0, windows = 0;
        for (int j = 0; j < count; ++j) {
            const cs_finish_job& job = jobs[j];
            if (job.frames <= 0)
                throw std::invalid_argument("cs_finish_natural_static: job " + std::to_string(j) + " has no frames");
            table.jobs[j] = job;
            frames += size_t(job.frames);
            if (frames > kMaxFrames)
                throw std::invalid_argument("cs_finish_natural_static: the jobs' " + std::to_string(frames) +
                                            "+ frames exceed the limit of " + std::to_string(kMaxFrames));
            blocks += (job.frames + kBlockFrames - 1) / kBlockFrames;
            windows += (job.frames + window - 1) / window;
        }
        unsigned char* scratch = scratchOnCurrentDevice();
        const auto s = static_cast<cudaStream_t>(stream);
        finishSetupKernel<<<1, kMaxJobs, 0, s>>>(table, reinterpret_cast<JobInfo*>(scratch + kJobsAt),
                                                  reinterpret_cast<int*>(scratch + kBlockJobAt),
                                                  reinterpret_cast<int*>(scratch + kWindowJobAt));

        BatchView view{};
        view.jobs = reinterpret_cast<const JobInfo*>(scratch + kJobsAt);
        view.blockJob = reinterpret_cast<const int*>(scratch + kBlockJobAt);
        view.windowJob = reinterpret_cast<const int*>(scratch + kWindowJobAt);
        view.mix = const_cast<float*>(mix);
        view.jobCount = count;
        FinishView finish{};
        finish.scans = reinterpret_cast<JobScan*>(scratch + kScansAt);
        finish.stereo = reinterpret_cast<StereoStats*>(scratch + kStereoAt);
        finish.windows = reinterpret_cast<MonoStats*>(scratch + kWindowsAt);
        finish.mono = reinterpret_cast<short*>(scratch + kMonoAt);
        finish.packed = packed;
        finish.results = results;
        finish.blockCount = blocks;
        finish.windowCount = windows;
        const TailConfig tail{window, 2 * rate, int(std::nearbyint(rate / 4.)), int(std::nearbyint(rate / 10.)),
                              std::pow(10., -1.5), 32768 * std::pow(10., -3.9), 32768 * std::pow(10., -3.)};
        launchScan(view, finish.stereo, blocks, s);
        launchFinish(view, finish, true, false, tail, s);
        const cudaError_t status = cudaGetLastError();
        if (status != cudaSuccess)
            throw std::runtime_error(std::string("static finishing launch: ") + cudaGetErrorString(status));
        return 0;
    } catch (const std::exception& error) {
        lastStaticError = error.what();
        return 1;
    }
}

extern "C" const char* cs_finish_natural_static_error(void) { return cs::lastStaticError.c_str(); }
