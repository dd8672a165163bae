// Host-side inputs of the render path: instruments (SFZ regions), MIDI event
// streams and the decoded sample bank.  These mirror the reference's
// src/sfz/instrument.h:15-136, src/io/midi.h:8-26 and src/io/audio.h:9-37, with
// the same defaults, because the planner's output must match the reference's
// bit for bit.
#pragma once

#include "../../include/claysampler_b200.h"

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace csh {

enum class Trigger { attack, release, releaseKey, first, legato };
enum class LoopMode { automatic, none, oneShot, continuous, sustain };
enum class OffMode { fast, normal, time };
enum class TailPolicy { natural, orig, custom };

struct Condition {
    uint8_t cc, low, high;
};

struct Crossfade {
    int inLow = 0, inHigh = 0, outLow = 127, outHigh = 127;
    bool power = true;
};

// A parameter driven by a controller: `depth` x curve(CC value).
struct Modulation {
    int target;                         // enum cs_mod_target
    int cc;
    float depth = 0;
    int curve = 0, smooth = 0;
};

struct Filter {
    int type = CS_FILTER_NONE;
    float cutoff = 0, resonance = 0, keyTrack = 0, velocityTrack = 0, random = 0;
    int keyCenter = 60;
};

struct Equalizer {
    float frequency = 0, bandwidth = 1, gain = 0;
    bool enabled = false;
};

struct Lfo {
    int wave = 0;
    float frequency = 0, phase = 0, delay = 0, fade = 0;
    std::map<int, float> depths;        // target -> depth
    std::vector<Modulation> modulation;
};

struct SecondaryEnvelope {
    std::array<float, 7> values{0, 0, 0, 0, 1, 0, 0};   // delay attack hold decay sustain start release
    std::array<float, 7> velocity{};
    float depth = 0, velocityDepth = 0;
    bool enabled = false, dynamic = false;
};

struct FlexPoint {
    float seconds = 0, level = 0;
    std::map<int, float> timeCC;
};

struct PitchEnvelope {
    std::map<int, FlexPoint> points;
    int sustain = -1;
    float depth = 0;
    std::map<int, float> depthCC;
};

struct Region {
    int sample = -1;
    int lowKey = 0, highKey = 127, rootKey = 60;
    int lowVelocity = 0, highVelocity = 127;
    int offset = 0, end = -1, loopStart = -1, loopEnd = -1;
    int transpose = 0;
    int sequenceLength = 1, sequencePosition = 1;
    int switchLow = -1, switchHigh = -1, switchDefault = -1;
    int switchDown = -1, switchUp = -1, switchPrevious = -1;
    int notePolyphony = 0;
    int sustainCC = 64, sustainLow = 1;
    int64_t group = 0, offBy = 0;
    bool sustainEnabled = true, releaseDead = false, switchRange = false, triggerOnNote = true;
    bool chokedByGroup = false, envelopeDynamic = false, selfMask = true;
    bool explicitSequencePosition = false;
    Trigger trigger = Trigger::attack;
    LoopMode loop = LoopMode::automatic;
    OffMode offMode = OffMode::fast;
    int generator = CS_GEN_NONE;
    float oscillatorPhase = 0;
    float volume = 0, amplitude = 1, velocityTrack = 1, pan = 0, width = 1, position = 0;
    float keyTrack = 100, tune = 0, bendUp = 200, bendDown = -200;
    int bendSmooth = 0;
    float delay = 0, envelopeDelay = 0, attack = 0, hold = 0, decay = 0, sustain = 1;
    float start = 0, release = 0.001f, releaseDecay = 0;
    float randomLow = 0, randomHigh = 1;
    float ampRandom = 0, pitchRandom = 0, offTime = .006f, loopCrossfade = .001f;
    Crossfade keyFade, velocityFade;
    std::map<int, Crossfade> controllerFades;
    bool powerControllerFade = true;
    std::vector<std::pair<int, float>> velocityCurve;
    std::vector<Condition> conditions;
    std::vector<Condition> ccTriggers;
    std::vector<Modulation> modulation;
    std::array<float, 7> velocityEnvelope{};
    std::array<Filter, 2> filters;
    std::array<Equalizer, 3> eq;
    std::map<int, Lfo> lfos;
    std::array<SecondaryEnvelope, 2> secondary;
    std::map<int, PitchEnvelope> pitchEnvelopes;
    int offsetRandom = 0;
};

using Curve = std::array<float, 128>;

struct Instrument {
    std::vector<Region> regions;
    std::array<std::vector<int>, 128> byKey;
    std::array<std::vector<int>, 128> byCC;
    std::array<bool, 128> switchKeys{};
    int initialSwitch = -1;
    bool hasOffBy = false;
    std::array<float, 128> initialCC = [] {
        std::array<float, 128> values{};
        values[7] = 100;
        values[10] = 63.5f;
        values[11] = 127;
        return values;
    }();
    std::array<bool, 128> usedCC{};
    std::map<int, float> extendedCCDefaults;
    std::map<int, Curve> curves;
};

enum class EventKind { on, off, control, bend };

struct Event {
    int frame;
    EventKind kind;
    int a, b;
};

struct Midi {
    std::vector<Event> events;
    int end = 0;
    int bodyFrames = 0;
    std::vector<int> onsets;
};

struct Sample {
    uint64_t offset;                    // UINT64_MAX until decoded
    int frames, rate, channels, loopFirst, loopEnd;
};

// Interleaved float32 sample bank (the reference's AudioBank, src/io/audio.h:18-37).
class SampleBank {
public:
    int describe(const std::string& path);
    const Sample& decode(int id);
    void releaseDecoded();
    std::vector<Sample> samples;
    std::vector<float> pcm;

private:
    std::map<std::string, int> loaded_;
    std::vector<std::string> paths_;
};

// The planned job (the reference's RenderPlan, src/render/plan.h:9-20).
struct Plan {
    std::vector<cs_voice_span> spans;
    std::vector<std::vector<cs_control_point>> controls;
    std::vector<cs_voice_modulation> modulation;
    int filterTracks = 0;
    int frames = 0;
    int musicEnd = 0, limit = 0, fadeFrames = 0;
    bool tailClipped = false;
    int bodyFrames = 0;
    std::vector<int> onsets;
    size_t volumeGroup = 0;
};

Instrument loadInstrument(const std::string& path, SampleBank& bank);
float curveValue(const Instrument& instrument, int curve, float value);
Midi loadMidi(const std::string& path, int rate, TailPolicy tail, bool measure);
Plan planRender(const Instrument& instrument, SampleBank& bank, const Midi& midi, int rate, unsigned seed, int limit,
                TailPolicy tail);

} // namespace csh
