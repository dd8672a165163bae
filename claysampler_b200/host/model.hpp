// Data model of the C++ host: what an SFZ instrument asks of a voice, a job's
// timed MIDI events, the decoded sample bank and the planned job handed to the
// renderer.
//
// A region is kept as a set of specifications grouped by concern (how it is
// selected, where its source comes from, its amplitude, pitch, envelope, voice
// rules, filters, modulators and controller bindings).  Keyed collections that
// the planner walks in key order (LFOs by index, LFO depths by target, controller
// crossfades by controller, flex envelopes and their stages by index) are sorted
// vectors: the walk order is part of the plan the renderer receives, and it
// follows the SFZ format's own numbering.  The defaults below are the SFZ
// format's (sfizz 1.2.3's, which the reference follows: src/sfz/instrument.h).
#pragma once

#include "../../include/claysampler_b200.h"

#include <algorithm>
#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace clayhost {

enum class Trigger { attack, release, releaseKey, first, legato };
enum class LoopKind { unset, off, oneShot, continuous, sustain };
enum class OffKind { fast, normal, time };
enum class TailPolicy { natural, orig, custom };

// Index of an envelope stage value (ampeg_*, fileg_*, pitcheg_*).
enum Stage { kDelay, kAttack, kHold, kDecay, kSustain, kStart, kRelease, kStages };

// A sorted vector used as a small ordered map: `slot` finds or inserts `key`.
template <class K, class V>
struct Keyed {
    std::vector<std::pair<K, V>> items;
    V& slot(const K& key)
    {
        auto at = std::lower_bound(items.begin(), items.end(), key,
                                   [](const std::pair<K, V>& item, const K& k) { return item.first < k; });
        if (at == items.end() || at->first != key)
            at = items.insert(at, {key, V{}});
        return at->second;
    }
    const V* find(const K& key) const
    {
        auto at = std::lower_bound(items.begin(), items.end(), key,
                                   [](const std::pair<K, V>& item, const K& k) { return item.first < k; });
        return at == items.end() || at->first != key ? nullptr : &at->second;
    }
    bool empty() const { return items.empty(); }
    auto begin() const { return items.begin(); }
    auto end() const { return items.end(); }
    auto begin() { return items.begin(); }
    auto end() { return items.end(); }
};

struct Range {
    int lo, hi;
    bool contains(int v) const { return v >= lo && v <= hi; }
};

struct CcRange {
    uint8_t cc, lo, hi;
};

// A controller (0-127), or one of the extended sources 131-141, driving a
// modulation target: depth x curve(value), optionally smoothed.
struct CcBinding {
    int target;                         // enum cs_mod_target
    int cc;
    float depth = 0;
    int curve = 0, smoothMs = 0;
};

struct Crossfade {
    int inLo = 0, inHi = 0, outLo = 127, outHi = 127;
    bool power = true;
};

// Which events start a voice of the region.
struct Selection {
    Trigger trigger = Trigger::attack;
    Range keys{0, 127};
    bool onNotes = true;                // false: only CC triggers start it
    int center = 60;                    // pitch_keycenter
    Range velocities{0, 127};
    float randomLo = 0, randomHi = 1;
    int sequenceLength = 1, sequencePosition = 1;
    bool sequenceExplicit = false;
    int switchLo = -1, switchHi = -1, switchDefault = -1;
    int switchDown = -1, switchUp = -1, switchPrevious = -1;
    bool switchIsRange = false;
    std::vector<CcRange> ccConditions;  // locc/hicc
    std::vector<CcRange> ccTriggers;    // on_locc/on_hicc
};

// Where the voice's source comes from.
struct Source {
    int sampleId = -1;                  // index in the bank, -1 for generators
    int generator = CS_GEN_NONE;
    float oscillatorPhase = 0;
    int offset = 0, offsetRandom = 0;
    int end = -1;                       // last frame + 1 once resolved
    LoopKind loop = LoopKind::unset;
    int loopStart = -1, loopEnd = -1;
    float loopCrossfade = .001f;        // seconds
};

struct Amplitude {
    float volumeDb = 0, linear = 1, velocityTrack = 1, randomDb = 0;
    std::vector<std::pair<int, float>> velocityCurve;
    float pan = 0, width = 1, position = 0;
    Crossfade keyFade, velocityFade;
    Keyed<int, Crossfade> ccFades;
    bool ccFadePower = true;
};

struct Pitch {
    float keyTrack = 100, tune = 0, random = 0, bendUp = 200, bendDown = -200;
    int transpose = 0, bendSmoothMs = 0;
};

// An envelope generator: stage values, their velocity tracking, and whether CC
// changes may retune it mid-voice.
struct EnvelopeSpec {
    std::array<float, kStages> stage{0, 0, 0, 0, 1, 0, .001f};
    std::array<float, kStages> perVelocity{};
    bool dynamic = false;
};

// Voice-level rules: choke groups, release handling, polyphony, pedals.
struct VoiceRules {
    int64_t group = 0, offBy = 0;
    bool chokedByGroup = false;
    OffKind offMode = OffKind::fast;
    float offTime = .006f;
    int notePolyphony = 0;
    bool selfMask = true;
    float releaseDecay = 0;
    bool releaseDead = false;
    bool pedal = true;
    int pedalCc = 64, pedalLow = 1;
    float delay = 0;
};

struct FilterSpec {
    int type = CS_FILTER_NONE;
    float cutoff = 0, resonance = 0, keyTrack = 0, velocityTrack = 0, random = 0;
    int keyCenter = 60;
};

struct EqSpec {
    float frequency = 0, bandwidth = 1, gain = 0;
    bool on = false;
};

struct LfoSpec {
    int wave = 0;
    float frequency = 0, phase = 0, delay = 0, fade = 0;
    Keyed<int, float> depth;            // target -> depth, in target order
    std::vector<CcBinding> ccs;         // in definition order
};

// fileg (slot 0) and pitcheg (slot 1).
struct AuxEnvelope {
    EnvelopeSpec shape{{0, 0, 0, 0, 1, 0, 0}, {}, false};
    float depth = 0, velocityDepth = 0;
    bool on = false;
};

struct FlexStage {
    float seconds = 0, level = 0;
    Keyed<int, float> secondsCc;
};

struct FlexEnvelope {
    Keyed<int, FlexStage> stages;
    int sustain = -1;
    float pitch = 0;
    Keyed<int, float> pitchCc;
};

struct Region {
    Selection select;
    Source source;
    Amplitude amp;
    Pitch pitch;
    EnvelopeSpec ampEnvelope;
    VoiceRules rules;
    std::array<FilterSpec, 2> filters;
    std::array<EqSpec, 3> eqs;
    Keyed<int, LfoSpec> lfos;           // by index; -1, -2, -3: pitchlfo, amplfo, fillfo
    std::array<AuxEnvelope, 2> aux;
    Keyed<int, FlexEnvelope> flex;      // egN
    std::vector<CcBinding> bindings;    // in definition order
};

using Curve = std::array<float, 128>;

struct Instrument {
    std::vector<Region> regions;
    std::array<std::vector<int>, 128> regionsByKey, regionsByCc;
    std::array<bool, 128> switchKey{};
    int startSwitch = -1;
    bool anyChoke = false;
    std::array<float, 128> startCc{};
    std::array<bool, 128> ccInUse{};
    std::map<int, float> extendedDefaults;
    std::map<int, Curve> curves;

    Instrument()
    {
        startCc[7] = 100;
        startCc[10] = 63.5f;
        startCc[11] = 127;
    }
};

// ---- MIDI ---------------------------------------------------------------------------

enum class EventType { noteOn, noteOff, control, bend };

struct TimedEvent {
    int frame;
    EventType type;
    int data1, data2;                   // key / controller / bend value, velocity / value
};

struct Score {
    std::vector<TimedEvent> events;
    int endFrame = 0;
    int bodyFrames = 0;                 // last note end (quality measurement)
    std::vector<int> onsets;            // distinct note starts, ascending
};

// ---- sample bank ----------------------------------------------------------------------

struct Sample {
    uint64_t offset;                    // UINT64_MAX until decoded
    int frames, rate, channels, loopFirst, loopEnd;
};

// Interleaved float32 samples, each decoded the first time a voice needs it, so
// offsets follow first use (the layout the renderer's bank upload receives).
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

// ---- planned job ------------------------------------------------------------------------

struct Plan {
    std::vector<cs_voice_span> spans;
    std::vector<std::vector<cs_control_point>> tracks;
    std::vector<cs_voice_modulation> bindings;
    int filterTracks = 0;
    int frames = 0;
    int musicEnd = 0, limit = 0, fadeFrames = 0;
    bool tailClipped = false;
    int bodyFrames = 0;
    std::vector<int> onsets;
    uint64_t volumeGroup = 0;
};

Instrument readInstrument(const std::string& path, SampleBank& bank);
float applyCurve(const Instrument& instrument, int curve, float value);
Score readScore(const std::string& path, int rate, TailPolicy tail, bool measure);
Plan planJob(const Instrument& instrument, SampleBank& bank, const Score& score, int rate, unsigned seed, int limit,
             TailPolicy tail);

} // namespace clayhost
