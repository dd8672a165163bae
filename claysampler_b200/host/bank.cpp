// Sample bank: WAV files decoded to one interleaved float32 array, each sample
// decoded the first time a region using it triggers, so offsets follow trigger
// order as in the reference's AudioBank (src/io/audio.cpp:93-154).
//
// Supported: RIFF/WAVE PCM 16/24/32-bit integer and 32-bit float, mono or stereo.
// Integers scale by 2^-(bits-1) (exact in float32, as libsndfile's normalised
// float read); a `smpl` chunk's first forward loop gives [start, end + 1).
#include "model.hpp"

#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <limits>
#include <stdexcept>

namespace clayhost {
namespace {

uint32_t le32(const unsigned char* p) { return uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16 | uint32_t(p[3]) << 24; }
uint16_t le16(const unsigned char* p) { return uint16_t(p[0] | p[1] << 8); }

struct WaveInfo {
    int64_t frames = 0;
    int rate = 0, channels = 0, bits = 0, loopFirst = 0, loopEnd = 0;
    bool isFloat = false;
    size_t dataOffset = 0;
};

std::vector<unsigned char> readFile(const std::string& path)
{
    std::ifstream file(path, std::ios::binary | std::ios::ate);
    if (!file)
        throw std::runtime_error("cannot decode mono or stereo sample " + path);
    const std::streamoff size = file.tellg();
    std::vector<unsigned char> data(size_t(size > 0 ? size : 0));
    file.seekg(0);
    if (!data.empty() && !file.read(reinterpret_cast<char*>(data.data()), std::streamsize(data.size())))
        throw std::runtime_error("cannot read sample " + path);
    return data;
}

WaveInfo parseWave(const std::vector<unsigned char>& data, const std::string& path)
{
    WaveInfo info;
    const auto fail = [&]() -> WaveInfo { throw std::runtime_error("cannot decode mono or stereo sample " + path); };
    if (data.size() < 12 || std::memcmp(data.data(), "RIFF", 4) || std::memcmp(data.data() + 8, "WAVE", 4))
        return fail();
    int format = 0;
    bool haveData = false;
    uint32_t dataBytes = 0;
    for (size_t pos = 12; pos + 8 <= data.size();) {
        const unsigned char* chunk = data.data() + pos;
        uint32_t length = le32(chunk + 4);
        if (pos + 8 + length > data.size())
            length = uint32_t(data.size() - pos - 8);
        if (!std::memcmp(chunk, "fmt ", 4) && length >= 16) {
            format = le16(chunk + 8);
            info.channels = le16(chunk + 10);
            info.rate = int(le32(chunk + 12));
            info.bits = le16(chunk + 22);
            if (format == 0xfffe && length >= 40)
                format = le16(chunk + 8 + 24);
        } else if (!std::memcmp(chunk, "data", 4)) {
            info.dataOffset = pos + 8;
            dataBytes = length;
            haveData = true;
        } else if (!std::memcmp(chunk, "smpl", 4) && length >= 60) {
            const uint32_t loops = le32(chunk + 8 + 28);
            if (loops > 0 && le32(chunk + 8 + 40) == 0) {
                info.loopFirst = int(le32(chunk + 8 + 44));
                info.loopEnd = int(le32(chunk + 8 + 48)) + 1;
            }
        }
        pos += 8 + length + (length & 1);
    }
    info.isFloat = format == 3;
    if (!haveData || (format != 1 && format != 3) || info.channels < 1 || info.rate <= 0 ||
        (info.isFloat ? info.bits != 32 : info.bits != 16 && info.bits != 24 && info.bits != 32))
        return fail();
    info.frames = int64_t(dataBytes) / (info.channels * (info.bits / 8));
    if (info.frames <= 0 || info.frames > std::numeric_limits<int>::max() || (info.channels != 1 && info.channels != 2))
        return fail();
    if (!(info.loopFirst < info.loopEnd && int64_t(info.loopEnd) <= info.frames))
        info.loopFirst = info.loopEnd = 0;
    return info;
}

} // namespace

int SampleBank::describe(const std::string& path)
{
    if (const auto it = loaded_.find(path); it != loaded_.end())
        return it->second;
    const std::string key = std::filesystem::weakly_canonical(std::filesystem::path(path)).string();
    if (const auto it = loaded_.find(key); it != loaded_.end()) {
        loaded_.emplace(path, it->second);
        return it->second;
    }
    const auto data = readFile(key);
    const WaveInfo info = parseWave(data, path);
    const int id = int(samples.size());
    samples.push_back({UINT64_MAX, int(info.frames), info.rate, info.channels, info.loopFirst, info.loopEnd});
    paths_.push_back(key);
    loaded_.emplace(key, id);
    if (path != key)
        loaded_.emplace(path, id);
    return id;
}

const Sample& SampleBank::decode(int id)
{
    Sample& sample = samples.at(size_t(id));
    if (sample.offset != UINT64_MAX)
        return sample;
    const std::string& path = paths_.at(size_t(id));
    const auto data = readFile(path);
    const WaveInfo info = parseWave(data, path);
    if (info.frames != sample.frames || info.rate != sample.rate || info.channels != sample.channels)
        throw std::runtime_error("sample changed since it was opened " + path);
    const size_t offset = pcm.size();
    const size_t count = size_t(info.frames) * size_t(info.channels);
    pcm.resize(offset + count);
    float* out = pcm.data() + offset;
    const unsigned char* p = data.data() + info.dataOffset;
    const int width = info.bits / 8;
    for (size_t i = 0; i < count; ++i, p += width) {
        float value;
        if (info.isFloat) {
            std::memcpy(&value, p, 4);
        } else if (width == 2) {
            value = float(int16_t(le16(p))) * (1.0f / 32768.0f);
        } else if (width == 3) {
            const int32_t v = int32_t(uint32_t(p[0]) << 8 | uint32_t(p[1]) << 16 | uint32_t(p[2]) << 24) >> 8;
            value = float(v) * (1.0f / 8388608.0f);
        } else {
            value = float(double(int32_t(le32(p))) * (1.0 / 2147483648.0));
        }
        if (!std::isfinite(value)) {
            pcm.resize(offset);
            throw std::runtime_error("invalid sample data in " + path);
        }
        out[i] = value;
    }
    sample.offset = offset;
    return sample;
}

void SampleBank::releaseDecoded()
{
    std::vector<float>().swap(pcm);
    for (auto& sample : samples)
        sample.offset = UINT64_MAX;
}

} // namespace clayhost
