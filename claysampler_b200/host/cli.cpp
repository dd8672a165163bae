// claysampler — the command line of the batch voice renderer.
//
// Keeps the reference CLI's surface (src/main.cpp): the same flags, the UTF-8
// `--jobs` manifest (group, SFZ, MIDI, output per line; paths relative to the
// manifest), the stdout protocol (DEVICE, INIT, OK, SKIP, QUALITY, VOLUME, PASS,
// TRANSFER), the stderr protocol (REJECT, ERROR) and the exit codes (0 all jobs
// written, 1 fatal error, 2 some job rejected).  Planning runs on this package's
// C++ planner (include/claysampler_host.h) one planning batch ahead of the GPU,
// rendering on the B200 renderer (include/claysampler_b200.h), and WAV writing on
// background tasks, as in the reference.
#include "../../include/claysampler_b200.h"
#include "../../include/claysampler_host.h"
#include "../csrc/plan_blob.hpp"

#include <algorithm>
#include <array>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <future>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <optional>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

using Path = std::filesystem::path;
using Clock = std::chrono::steady_clock;

double since(Clock::time_point start) { return std::chrono::duration<double>(Clock::now() - start).count(); }

enum class Tail { natural = 0, orig = 1, custom = 2 };

struct Options {
    Path sfz, output, jobs;
    int device = 0, rate = 44100, passes = 1;
    size_t cpuBatchJobs = 64, gpuBatchJobs = 64;
    Tail tail = Tail::natural;
    std::optional<double> tailMax, maxAudio;
    std::optional<int> tailFadeMs;
    std::vector<Path> midi;
    std::string quality = "off";
    std::vector<std::pair<std::string, std::string>> thresholds;
    std::string outputFormat = "wav";
    int flacLevel = 5;
    bool resume = false, groupVolume = false;
    std::optional<int> groupMinimum, waitingMiB;
};

int parseInt(const std::string& text, long long low, long long high)
{
    size_t used = 0;
    long long value = 0;
    try {
        value = std::stoll(text, &used);
    } catch (const std::exception&) {
        used = 0;
    }
    if (text.empty() || used != text.size() || value < low || value > high)
        throw std::runtime_error("invalid numeric argument " + text);
    return int(value);
}

double parseNumber(const std::string& text, double low, double high)
{
    size_t used = 0;
    double value = 0;
    try {
        value = std::stod(text, &used);
    } catch (const std::exception&) {
        used = 0;
    }
    if (text.empty() || used != text.size() || !std::isfinite(value) || value < low || value > high)
        throw std::runtime_error("invalid numeric argument " + text);
    return value;
}

Options parseOptions(int argc, char** argv)
{
    Options o;
    for (int i = 1; i < argc; ++i) {
        const std::string name = argv[i];
        if (name.empty() || name[0] != '-') {
            o.midi.emplace_back(name);
            continue;
        }
        if (name == "--resume") {
            o.resume = true;
            continue;
        }
        if (i + 1 == argc)
            throw std::runtime_error("missing value for " + name);
        const std::string value = argv[++i];
        if (name == "--sfz") o.sfz = value;
        else if (name == "--output") o.output = value;
        else if (name == "--output-format") {
            if (value != "wav" && value != "flac")
                throw std::runtime_error("expected --output-format wav or flac");
            o.outputFormat = value;
        } else if (name == "--flac-level") o.flacLevel = parseInt(value, 0, 8);
        else if (name == "--jobs") o.jobs = value;
        else if (name == "--nvrtc" || name == "--sndfile") {
            // Accepted for compatibility: kernels are compiled offline and samples are
            // decoded without libsndfile.
        } else if (name == "--device") o.device = parseInt(value, 0, 1024);
        else if (name == "--samplerate") o.rate = parseInt(value, 8000, 192000);
        else if (name == "--passes") o.passes = parseInt(value, 1, 1000);
        else if (name == "--cpu-batch-jobs") o.cpuBatchJobs = size_t(parseInt(value, 1, INT_MAX));
        else if (name == "--gpu-batch-jobs") o.gpuBatchJobs = size_t(parseInt(value, 1, INT_MAX));
        else if (name == "--tail-policy") {
            if (value == "natural") o.tail = Tail::natural;
            else if (value == "orig") o.tail = Tail::orig;
            else if (value == "custom") o.tail = Tail::custom;
            else throw std::runtime_error("expected --tail-policy natural, orig, or custom");
        } else if (name == "--tail-max-seconds") o.tailMax = parseNumber(value, 0, 3600);
        else if (name == "--tail-fade-ms") o.tailFadeMs = parseInt(value, 0, 3600000);
        else if (name == "--max-audio-seconds") o.maxAudio = parseNumber(value, 0, 3600);
        else if (name == "--quality-gate") o.quality = value;
        else if (name.rfind("--qa-", 0) == 0) {
            for (const auto& [seen, _] : o.thresholds)
                if (seen == name)
                    throw std::runtime_error("duplicate option " + name);
            o.thresholds.emplace_back(name, value);
        } else if (name == "--group-volume") {
            if (value != "off" && value != "mean")
                throw std::runtime_error("expected --group-volume off or mean");
            o.groupVolume = value == "mean";
        } else if (name == "--group-min-members") o.groupMinimum = parseInt(value, 2, 100000);
        else if (name == "--group-wait-mib") o.waitingMiB = parseInt(value, 0, 16384);
        else throw std::runtime_error("unknown option " + name);
    }
    const bool manifest = !o.jobs.empty();
    if (!manifest && (o.sfz.empty() || o.output.empty() || o.midi.empty()))
        throw std::runtime_error("provide --sfz, --output, and at least one MIDI path");
    if (manifest && (!o.sfz.empty() || !o.output.empty() || !o.midi.empty()))
        throw std::runtime_error("--jobs supplies the SFZ, MIDI and output paths");
    if (o.quality != "off" && o.quality != "clayengine" && o.quality != "custom")
        throw std::runtime_error("expected --quality-gate off, clayengine, or custom");
    if (o.quality != "custom" && !o.thresholds.empty())
        throw std::runtime_error("quality thresholds require --quality-gate custom");
    if (o.groupVolume && !manifest)
        throw std::runtime_error("--group-volume mean requires --jobs");
    if (!o.groupVolume && (o.groupMinimum || o.waitingMiB))
        throw std::runtime_error("group options require --group-volume mean");
    if (o.tail == Tail::custom && !o.tailMax)
        throw std::runtime_error("custom tail requires --tail-max-seconds");
    if (o.tail != Tail::custom && (o.tailMax || o.tailFadeMs))
        throw std::runtime_error("tail length and fade options require --tail-policy custom");
    if (o.maxAudio && o.tail != Tail::natural)
        throw std::runtime_error("--max-audio-seconds requires --tail-policy natural");
    if (o.outputFormat == "flac")
        throw std::runtime_error("FLAC output needs libsndfile's encoder, which this build does not include");
    return o;
}

// The quality gate's thresholds: ClayEngine's defaults, then --qa-* overrides
// (the reference's audioConfig, src/main.cpp:169-187).
cs_audio_config audioConfig(const Options& o)
{
    const auto power = [](double dbfs) { return 4294967296. * std::pow(10., dbfs / 10); };
    cs_audio_config c{};
    c.rate = o.rate;
    c.window = int(std::nearbyint(o.rate / 20.));
    c.maxFrames = 375 * o.rate;
    c.minPeak = 32;
    c.enabled = o.quality != "off";
    c.minMedian = -38;
    c.minQuartile = -45;
    c.silencePower = power(-70);
    c.maxSilentFraction = .75;
    c.maxSilentFrames = 10. * o.rate;
    c.maxClippedFraction = .0001;
    for (const auto& [name, value] : o.thresholds) {
        if (name == "--qa-max-seconds") c.maxFrames = int(std::floor(parseNumber(value, 0, 3600) * o.rate));
        else if (name == "--qa-min-peak") c.minPeak = parseInt(value, 0, 32768);
        else if (name == "--qa-min-onset-median-dbfs") c.minMedian = parseNumber(value, -120, 0);
        else if (name == "--qa-min-onset-quartile-dbfs") c.minQuartile = parseNumber(value, -120, 0);
        else if (name == "--qa-silence-dbfs") c.silencePower = power(parseNumber(value, -120, 0));
        else if (name == "--qa-max-silence-fraction") c.maxSilentFraction = parseNumber(value, 0, 1);
        else if (name == "--qa-max-silence-seconds") c.maxSilentFrames = parseNumber(value, 0, 3600) * o.rate;
        else if (name == "--qa-max-clipped-fraction") c.maxClippedFraction = parseNumber(value, 0, 1);
        else throw std::runtime_error("unknown option " + name);
    }
    return c;
}

struct Task {
    Path sfz, midi, output;
    uint64_t group = 0;
};

// Jobs in render order.  In a manifest, a volume group takes the slot of its first
// member and collects its later members there (src/main.cpp:194-262).
std::vector<Task> readTasks(const Options& o)
{
    std::vector<Task> tasks;
    if (o.jobs.empty()) {
        for (const auto& midi : o.midi) {
            Path name = midi.stem();
            name += "." + o.outputFormat;
            tasks.push_back({o.sfz, midi, o.output / name, 0});
        }
    } else {
        std::ifstream file(o.jobs, std::ios::binary);
        if (!file)
            throw std::runtime_error("cannot open job manifest " + o.jobs.string());
        const Path root = std::filesystem::absolute(o.jobs).parent_path();
        std::map<std::string, size_t> slotOf;
        std::vector<std::vector<Task>> slots;
        size_t number = 0;
        for (std::string line; std::getline(file, line);) {
            if (++number == 1 && line.rfind("\xef\xbb\xbf", 0) == 0)
                line.erase(0, 3);
            if (!line.empty() && line.back() == '\r')
                line.pop_back();
            if (line.empty())
                continue;
            std::vector<std::string> column;
            for (size_t start = 0;;) {
                const size_t tab = line.find('\t', start);
                column.push_back(line.substr(start, tab == std::string::npos ? std::string::npos : tab - start));
                if (tab == std::string::npos)
                    break;
                start = tab + 1;
            }
            for (size_t c = 0; c < 4; ++c)
                if (c >= column.size() || column[c].empty())
                    throw std::runtime_error("expected group, SFZ, MIDI and output on manifest line " +
                                             std::to_string(number));
            if (column.size() > 4)
                throw std::runtime_error("invalid job manifest line " + std::to_string(number));
            if (line.find('\0') != std::string::npos)
                throw std::runtime_error("invalid job manifest line " + std::to_string(number));
            Task task{root / std::filesystem::u8path(column[1]), root / std::filesystem::u8path(column[2]),
                      root / std::filesystem::u8path(column[3]), 0};
            if (task.output.extension() != "." + o.outputFormat)
                throw std::runtime_error("expected a ." + o.outputFormat + " output on manifest line " +
                                         std::to_string(number));
            if (o.groupVolume && column[0] != "-") {
                const auto found = slotOf.emplace(column[0], slots.size());
                if (found.second)
                    slots.emplace_back();
                task.group = found.first->second + 1;
                slots[found.first->second].push_back(std::move(task));
            } else {
                slots.push_back({std::move(task)});
            }
        }
        if (!file.eof())
            throw std::runtime_error("cannot read job manifest " + o.jobs.string());
        for (auto& slot : slots)
            for (auto& task : slot)
                tasks.push_back(std::move(task));
    }
    if (tasks.empty())
        throw std::runtime_error("job manifest is empty");
    std::set<Path> outputs;
    for (const auto& task : tasks)
        if (!outputs.insert(std::filesystem::weakly_canonical(std::filesystem::absolute(task.output))).second)
            throw std::runtime_error("duplicate output path " + task.output.string());
    return tasks;
}

const char* statusText(int status)
{
    switch (status) {
    case CS_TAIL_OK: return nullptr;
    case CS_TAIL_DURATION: return "natural tail exceeded the tail or audio duration limit";
    case CS_TAIL_NONFINITE: return "natural render produced non-finite audio";
    case CS_TAIL_PEAK: return "excessive_peak: natural render requires more than 5 dB attenuation";
    case CS_TAIL_AUDIO_DURATION: return "rendered_audio_too_long";
    case CS_TAIL_QUIET_PERFORMANCE: return "quiet_performance";
    case CS_TAIL_EXCESSIVE_SILENCE: return "excessive_audio_silence";
    case CS_TAIL_SILENT_AUDIO: return "effectively_silent_audio";
    case CS_TAIL_CLIPPING: return "excessive_audio_clipping";
    case CS_TAIL_SILENT_BODY: return "silent_melody_body";
    case CS_TAIL_INCOMPLETE_GROUP: return "insufficient_qualified_group_members";
    case CS_TAIL_SCRATCH_MEMORY: return "CUDA mapped scratch allocation: out of memory";
    }
    return "unknown CUDA tail status";
}

// The planner, one instance for the whole run (instruments and the decoded bank
// persist across planning batches).
struct Host {
    cs_host* handle = nullptr;
    Host()
    {
        if (cs_host_create(&handle))
            throw std::runtime_error(cs_host_last_error());
    }
    ~Host() { cs_host_destroy(handle); }
    size_t bankFloats() const
    {
        const float* pcm = nullptr;
        size_t floats = 0;
        cs_host_bank(handle, &pcm, &floats);
        return floats;
    }
};

struct Image {
    void* data = nullptr;
    size_t size = 0;
    Image() = default;
    Image(const Image&) = delete;
    Image(Image&& other) noexcept : data(other.data), size(other.size) { other.data = nullptr; }
    ~Image() { cs_host_free(data); }
};

struct PlannedBatch {
    std::vector<Image> images;
    std::vector<cs_plan> plans;
    std::shared_ptr<std::vector<const Task*>> jobs = std::make_shared<std::vector<const Task*>>();
    std::vector<std::string> rejected;
    size_t next = 0;
    double seconds = 0;
    bool fresh = false;
};

// planBatch (src/main.cpp:298-361): up to --cpu-batch-jobs jobs, about 24 Mi
// frames, or the sample budget, without leaving a volume group half planned.
PlannedBatch planBatch(const Options& o, const std::vector<Task>& tasks, Host& host, size_t first,
                       size_t sampleBudget, bool fresh)
{
    const auto start = Clock::now();
    PlannedBatch batch;
    batch.fresh = fresh;
    if (fresh && cs_host_release_bank(host.handle))
        throw std::runtime_error(cs_host_last_error());
    const size_t count = std::min(o.cpuBatchJobs, tasks.size() - first);
    const bool manifest = !o.jobs.empty();
    size_t frames = 0;
    for (batch.next = first; batch.next < tasks.size(); ++batch.next) {
        const Task& task = tasks[batch.next];
        const bool continuesGroup = task.group && batch.next > first && tasks[batch.next - 1].group == task.group;
        if (!continuesGroup && (batch.next - first >= count || frames >= size_t(24) << 20 ||
                                (batch.next > first && host.bankFloats() >= sampleBudget / sizeof(float))))
            break;
        Image image;
        if (cs_host_plan(host.handle, task.sfz.c_str(), task.midi.c_str(), o.rate, int(o.tail),
                         o.maxAudio ? *o.maxAudio : -1.0, o.tailMax ? *o.tailMax : -1.0,
                         o.tailFadeMs ? *o.tailFadeMs : -1, o.quality != "off", o.groupVolume, task.group,
                         &image.data, &image.size)) {
            const Path& label = manifest ? task.output : task.midi;
            batch.rejected.push_back("REJECT\t" + label.string() + '\t' + cs_host_last_error() + '\n');
            continue;
        }
        batch.plans.push_back(cs::readPlanBlob(static_cast<const unsigned char*>(image.data), image.size));
        frames += size_t(batch.plans.back().frames);
        batch.images.push_back(std::move(image));
        batch.jobs->push_back(&task);
    }
    batch.seconds = since(start);
    return batch;
}

// A finished batch, owned by the writers.
struct Finished {
    std::vector<int16_t> pcm;
    std::vector<cs_tail_result> results;
};

struct Written {
    size_t passed = 0;
    std::string ok, rejected;
};

// writeBatch (src/main.cpp:384-433): QUALITY, VOLUME and OK lines, WAV output.
Written writeJobs(const Finished& batch, const std::vector<const Task*>& jobs, size_t begin, const Options& o,
                  int channels, bool manifest)
{
    std::ostringstream ok, rejected;
    Written out;
    for (size_t i = 0; i < jobs.size(); ++i) {
        const cs_tail_result& result = batch.results[begin + i];
        const Path& path = jobs[i]->output;
        const cs_audio_metrics& stats = result.audio;
        const char* failure = statusText(result.status);
        if (stats.measured) {
            const char* verdict = statusText(stats.verdict);
            ok << "QUALITY\t" << path.string() << '\t' << (verdict ? verdict : "accepted") << '\t' << result.frames
               << '\t' << stats.median << '\t' << stats.quartile << '\t' << stats.silentFraction << '\t'
               << double(stats.longestSilence) / o.rate << '\t' << stats.clippedFraction << '\n';
        }
        try {
            if (failure)
                throw std::runtime_error(failure);
            if (result.last < 0 && stats.gain <= 0)
                throw std::runtime_error("rendered audio is silent " + path.string());
            if (manifest)
                std::filesystem::create_directories(path.parent_path());
            const int16_t* pcm = batch.pcm.data() + result.offset * uint64_t(channels);
            if (cs_write_wave(path.c_str(), pcm, result.dataFrames, result.frames, o.rate, channels))
                throw std::runtime_error(cs_host_last_error());
            if (stats.gain > 0)
                ok << "VOLUME\t" << path.string() << '\t' << stats.bodyRms << '\t' << stats.targetRms << '\t'
                   << 20 * std::log10(stats.gain) << '\n';
            ok << "OK\t" << (manifest ? path : path.filename()).string() << '\t' << result.frames << '\t'
               << result.peak << '\t' << result.first << '\t' << result.last << '\n';
            ++out.passed;
        } catch (const std::exception& error) {
            rejected << "REJECT\t" << path.string() << '\t' << error.what() << '\n';
        }
    }
    out.ok = ok.str();
    out.rejected = rejected.str();
    return out;
}

struct Renderer {
    cs_renderer* handle = nullptr;
    Renderer(const Options& o, bool natural, const cs_audio_config& audio)
    {
        const int minimum = o.groupVolume ? o.groupMinimum.value_or(2) : 0;
        const size_t waiting = size_t(o.waitingMiB.value_or(256)) << 20;
        if (cs_renderer_create(o.device, natural, &audio, minimum, waiting, o.gpuBatchJobs, &handle))
            throw std::runtime_error(cs_last_error());
    }
    ~Renderer() { cs_renderer_destroy(handle); }
};

// One pass's rendering of one planned batch: publish -> writers.
struct Publisher {
    const Options& options;
    PlannedBatch& batch;
    std::deque<std::future<Written>>& writers;
    size_t& passed;
    double& kernelSeconds;
    int channels;
    bool manifest;

    void drain()
    {
        auto pending = std::move(writers.front());
        writers.pop_front();
        const Written written = pending.get();
        passed += written.passed;
        std::cout << written.ok << std::flush;
        std::cerr << written.rejected << std::flush;
    }

    static void callback(void* user, const cs_batch* b, size_t first)
    {
        static_cast<Publisher*>(user)->publish(*b, first);
    }

    void publish(const cs_batch& b, size_t first)
    {
        kernelSeconds += b.kernel_seconds;
        if (b.failed_scratch_bytes) {
            const Task& job = *(*batch.jobs)[first];
            std::cerr << "REJECT\t" << job.output.string() << '\t' << statusText(CS_TAIL_SCRATCH_MEMORY)
                      << " (bytes=" << b.failed_scratch_bytes << ")\tMIDI=" << job.midi.string()
                      << "\tSFZ=" << job.sfz.string() << '\n';
            return;
        }
        auto finished = std::make_shared<Finished>();
        finished->pcm.assign(b.pcm, b.pcm + b.pcm_samples);
        finished->results.assign(b.results, b.results + b.result_count);
        if (writers.size() >= 3)
            drain();
        std::vector<const Task*> jobs;
        for (size_t i = 0; i < b.result_count; ++i)
            jobs.push_back((*batch.jobs)[b.job_index_count ? b.job_indices[i] : first + i]);
        const Options* o = &options;
        const int ch = channels;
        const bool m = manifest;
        writers.push_back(std::async(std::launch::async, [finished, jobs = std::move(jobs), o, ch, m] {
            return writeJobs(*finished, jobs, 0, *o, ch, m);
        }));
    }
};

int run(const Options& o)
{
    const bool natural = o.tail == Tail::natural;
    const bool manifest = !o.jobs.empty();
    const int channels = natural ? 1 : 2;
    const cs_audio_config audio = audioConfig(o);
    std::vector<Task> tasks = readTasks(o);
    const auto start = Clock::now();
    if (o.resume) {
        // A group is skipped only when every member's output is complete
        // (src/main.cpp:444-457).
        std::vector<Task> pending;
        for (size_t first = 0, end; first < tasks.size(); first = end) {
            end = first + 1;
            while (tasks[first].group && end < tasks.size() && tasks[end].group == tasks[first].group)
                ++end;
            bool complete = true;
            for (size_t i = first; i < end && complete; ++i)
                complete = cs_wave_complete(tasks[i].output.c_str(), o.rate, channels) != 0;
            for (size_t i = first; i < end; ++i) {
                if (complete)
                    std::cout << "SKIP\t" << tasks[i].output.string() << '\n';
                else
                    pending.push_back(std::move(tasks[i]));
            }
        }
        tasks = std::move(pending);
        if (tasks.empty())
            return 0;
    }
    Host host;
    const size_t unlimited = std::numeric_limits<size_t>::max();
    const auto prefetch = [&](size_t next, size_t budget, bool fresh) {
        return std::async(std::launch::async, [&, next, budget, fresh] {
            return planBatch(o, tasks, host, next, budget, fresh);
        });
    };
    auto opening = prefetch(0, manifest ? size_t(512) << 20 : unlimited, false);
    Renderer renderer(o, natural, audio);
    PlannedBatch startup = opening.get();
    const size_t sampleBudget = manifest ? cs_sample_cache_budget(renderer.handle) : unlimited;
    const auto rotate = [&] { return manifest && host.bankFloats() >= sampleBudget / sizeof(float); };
    std::cout << "DEVICE\t" << cs_renderer_device(renderer.handle) << '\n' << "INIT\t" << since(start) << '\n';
    if (!manifest)
        std::filesystem::create_directories(o.output);
    size_t passed = 0;
    for (int pass = 1; pass <= o.passes; ++pass) {
        const auto passStart = Clock::now();
        double preparation = 0, kernelSeconds = 0;
        passed = 0;
        const size_t spilledBefore = cs_spilled_bytes(renderer.handle);
        const size_t downloadedBefore = cs_downloaded_bytes(renderer.handle);
        PlannedBatch batch = pass == 1 ? std::move(startup) : planBatch(o, tasks, host, 0, sampleBudget, rotate());
        std::deque<std::future<Written>> writers;
        for (;;) {
            for (const auto& line : batch.rejected)
                std::cerr << line;
            const auto uploadStart = Clock::now();
            if (!batch.plans.empty() || batch.fresh) {
                const float* pcm = nullptr;
                size_t floats = 0;
                cs_host_bank(host.handle, &pcm, &floats);
                if (cs_upload_samples(renderer.handle, pcm, floats, batch.fresh))
                    throw std::runtime_error(cs_last_error());
            }
            preparation += batch.seconds + since(uploadStart);
            // The next planning batch may grow the host bank, so it starts only after
            // this batch's samples are on the device.
            std::future<PlannedBatch> next;
            if (batch.next < tasks.size())
                next = prefetch(batch.next, sampleBudget, rotate());
            Publisher publisher{o, batch, writers, passed, kernelSeconds, channels, manifest};
            if (!batch.plans.empty() &&
                cs_render_window(renderer.handle, batch.plans.data(), batch.plans.size(), Publisher::callback,
                                 nullptr, &publisher))
                throw std::runtime_error(cs_last_error());
            // The batch's plans stay alive until its writers have copied what they need
            // (the published PCM and results are copied in the callback).
            if (!next.valid())
                break;
            batch = next.get();
        }
        Publisher drainer{o, batch, writers, passed, kernelSeconds, channels, manifest};
        while (!writers.empty())
            drainer.drain();
        std::cout << "PASS\t" << pass << '\t' << since(passStart) << '\t' << passed << '\t'
                  << cs_peak_bytes(renderer.handle) << '\t' << preparation << '\t' << kernelSeconds << '\n';
        if (audio.enabled || o.groupVolume)
            std::cout << "TRANSFER\t" << pass << '\t' << cs_downloaded_bytes(renderer.handle) - downloadedBefore
                      << '\t' << cs_spilled_bytes(renderer.handle) - spilledBefore << '\t'
                      << cs_peak_waiting_bytes(renderer.handle) << '\n';
    }
    return passed == tasks.size() ? 0 : 2;
}

int checkPresets(int argc, char** argv)
{
    int first = 2;
    if (argc > 3 && std::string(argv[first]) == "--sndfile")
        first += 2;
    if (first == argc)
        throw std::runtime_error("provide at least one SFZ path after --check-sfz");
    bool rejected = false;
    for (int i = first; i < argc; ++i) {
        int regions = 0;
        if (cs_host_check_sfz(argv[i], &regions)) {
            rejected = true;
            std::cout << "SFZ\tREJECT\t" << cs_host_last_error() << '\n';
        } else {
            std::cout << "SFZ\tOK\t" << regions << '\n';
        }
    }
    return rejected ? 2 : 0;
}

} // namespace

int main(int argc, char** argv)
{
    try {
        if (argc == 2 && std::string(argv[1]) == "--help") {
            std::cout << "Usage: claysampler --sfz preset.sfz --output directory [options] file.mid ...\n"
                         "       claysampler --jobs tasks.tsv [options]\n"
                         "Options: --output-format wav --resume\n"
                         "         --samplerate Hz --device index --passes count\n"
                         "         --cpu-batch-jobs count --gpu-batch-jobs count (default 64 each)\n"
                         "         --tail-policy natural|orig|custom (default natural)\n"
                         "         --max-audio-seconds seconds (natural)\n"
                         "         --tail-max-seconds seconds [--tail-fade-ms milliseconds] (custom)\n"
                         "         --quality-gate off|clayengine|custom (default off)\n"
                         "         --group-volume off|mean (default off; mean uses groups in --jobs)\n"
                         "         --group-min-members count --group-wait-mib MiB\n"
                         "       claysampler --check-sfz preset.sfz ...\n";
            return 0;
        }
        if (argc > 1 && std::string(argv[1]) == "--check-sfz")
            return checkPresets(argc, argv);
        return run(parseOptions(argc, argv));
    } catch (const std::exception& error) {
        std::cerr << "ERROR\t" << error.what() << '\n';
        return 1;
    }
}
