// The planner: an instrument and a job's timed MIDI events -> voice spans, control
// tracks and modulation bindings (the plan the renderer receives).
//
// It is organised as four cooperating parts:
//  * TrackBook   the plan's control tracks: MIDI controller automation (ramped
//                at the format's 1024-frame block and smoothed in 16-frame
//                steps), bend and crossfade tracks, memoised by what defines them;
//  * VoiceFactory turns (region, note, cause) into a voice span: source position,
//                pitch, envelopes, filters, gains, and the bindings that modulate it;
//  * LfoBaker    collects LFOs while voices start and bakes their output tracks once
//                every voice's end is known;
//  * Performer   walks the events: note on/off with round robins, key switches and
//                random layers, release triggers, pedals (sustain, sostenuto),
//                choke groups, per-note polyphony, pitch bend segments, controller
//                changes and CC triggers, emitting spans as voices end or change.
//
// The plan must be byte-identical to the reference planner's
// (src/render/plan.cpp): the same float expressions in the same order, the same
// random draws in the same sequence, spans emitted in the same order.  Those are
// the algorithm; the decomposition here is this host's own.
#include "model.hpp"

#include <climits>
#include <cmath>
#include <random>
#include <stdexcept>
#include <tuple>

namespace clayhost {
namespace {

constexpr int kForever = INT_MAX;
constexpr float kSilence = 1e-4f;           // a releasing voice fades out below this level
constexpr int kBendBlock = 1024;            // controller ramps start at their 1024-frame block
constexpr float kMasterDb = -7.35f;         // master gain of the non-natural policies

using Points = std::vector<cs_control_point>;

[[noreturn]] void fail(const std::string& message) { throw std::runtime_error(message); }

float uniform24(std::mt19937& g) { return std::generate_canonical<float, 24>(g); }

// Piecewise-linear value of a track at `frame` (the point at or before it).
float valueAt(const Points& track, int frame)
{
    const auto after = std::upper_bound(track.begin(), track.end(), frame,
                                        [](int f, const cs_control_point& p) { return f < p.frame; });
    const cs_control_point& p = after == track.begin() ? track.front() : *std::prev(after);
    return p.value + (frame - p.frame) * p.step;
}

// ---- envelope arithmetic shared with the renderer --------------------------------------

template <class Shape>
float levelAt(const Shape& e, int frame)
{
    if (e.releaseStart >= 0 && frame >= e.releaseStart) {
        if (frame >= e.fadeStart)
            return std::max(0.f, e.fadeValue - (frame - e.fadeStart + 1) * e.fadeStep);
        return e.releaseValue * std::exp((frame - e.releaseStart + 1) * e.releaseRate);
    }
    if (frame < e.attackStart)
        return e.start;
    if (frame < e.holdStart)
        return std::min(1.f, e.start + (frame - e.attackStart + 1) * e.attackStep);
    if (frame < e.decayStart)
        return 1;
    if (e.decayRate == 0)
        return e.sustain;
    return std::max(e.sustain, std::exp((frame - e.decayStart + 1) * e.decayRate));
}

// Release from `level` at `frame` over `seconds` (-80 dB), then a 50 ms linear fade.
template <class Shape>
void startReleaseCurve(Shape& e, int frame, int rate, float level, float seconds)
{
    e.releaseStart = frame;
    e.releaseValue = level;
    e.releaseRate = -9 / (std::clamp(seconds, .006f, 100.f) * rate);
    const int duration = level > kSilence ? static_cast<int>(std::log(kSilence / level) / e.releaseRate) : 0;
    e.fadeStart = frame + duration;
    e.fadeValue = level * std::exp(e.releaseRate * duration);
    e.fadeStep = std::max(kSilence, e.fadeValue) / (rate * .05f);
}

// Source frames a span moves through in its first `frames` frames, at its lowest
// pitch (the bound used for its end).
double travelled(const cs_voice_span& v, int frames)
{
    if (v.pitchSlope == 0)
        return v.step * v.minimumPitchRatio * frames;
    return v.step * v.minimumPitchRatio * std::expm1(v.pitchSlope * frames) / std::expm1(v.pitchSlope);
}

double wrapped(const cs_voice_span& v, double position)
{
    if (v.loopEnd > 0 && position >= v.loopEnd)
        return v.loopFirst + std::fmod(position - v.loopFirst, v.loopEnd - v.loopFirst);
    return position;
}

// The frame at which a span runs out of sample (unlooped samples), bounded by its
// envelope's end.
int spanEnd(const cs_voice_span& v, int envelopeEnd)
{
    if (v.loopEnd > 0 || v.generator != CS_GEN_NONE)
        return envelopeEnd;
    const int rampFrames = std::max(0, v.bendEnd - v.begin);
    const double rampTravel = travelled(v, rampFrames);
    const double remaining = v.sourceEnd - v.position;
    const double step = v.step * v.minimumPitchRatio;
    const double length = rampFrames && v.pitchSlope != 0 && remaining <= rampTravel
        ? std::ceil(std::log1p(std::max(0., remaining) * std::expm1(v.pitchSlope) / step) / v.pitchSlope)
        : rampFrames + std::ceil((remaining - rampTravel) / (step * std::exp(v.pitchSlope * rampFrames)));
    if (length > kForever - v.begin)
        return envelopeEnd;
    return std::min(envelopeEnd, v.begin + std::max(0, static_cast<int>(length)));
}

float lfoShape(int wave, double phase)
{
    const auto p = static_cast<float>(phase - std::floor(phase));
    switch (wave) {
    case 0: return p < .25f ? 4 * p : p > .75f ? 4 * p - 4 : 2 - 4 * p;     // triangle
    case 1: {                                                                // sine-like parabola
        const float x = 2 * p - 1;
        return -4 * x * (1 - std::abs(x));
    }
    case 2: return p < .75f;            // pulses of 75, 50, 25 and 12.5 %
    case 3: return p < .5f;
    case 4: return p < .25f;
    case 5: return p < .125f;
    case 6: return 2 * p - 1;           // saw up
    case 7: return 1 - 2 * p;           // saw down
    default: return 0;
    }
}

float velocityGain(const Region& r, int velocity)
{
    const float normalized = float(velocity) / 127;
    float gain = normalized * normalized;
    const auto& curve = r.amp.velocityCurve;
    if (!curve.empty()) {
        const auto hi = std::lower_bound(curve.begin(), curve.end(), velocity,
                                         [](const auto& point, int v) { return point.first < v; });
        if (hi->first == velocity) {
            gain = hi->second;
        } else {
            const auto lo = std::prev(hi);
            const float phase = float(velocity - lo->first) / (hi->first - lo->first);
            gain = lo->second + phase * (hi->second - lo->second);
        }
    }
    const float track = std::abs(r.amp.velocityTrack) * (1 - gain);
    return r.amp.velocityTrack < 0 ? track : 1 - track;
}

float crossfade(const Crossfade& xf, float value, bool controllerScale)
{
    const auto top = [controllerScale](int high) { return controllerScale && high == 127 ? 126 : high; };
    const int inHi = top(xf.inHi), outHi = top(xf.outHi);
    float up = 1, down = 1;
    if (value < xf.inLo)
        up = 0;
    else if (inHi > xf.inLo)
        up = std::min(1.f, float(value - xf.inLo) / (inHi - xf.inLo));
    if (outHi > xf.outLo)
        down = std::clamp(float(outHi - value) / (outHi - xf.outLo), 0.f, 1.f);
    return xf.power ? std::sqrt(up * down) : up * down;
}

// ---- control tracks ------------------------------------------------------------------------

// A MIDI controller (or, as controller 128, the pitch bend) as a control track:
// each change ramps linearly from its 1024-frame block to the event (the format's
// block-wise interpolation), a reset (CC121) returns to `initial`, and with
// `smoothFrames` >= 2 the result is followed in 16-frame steps by a slew toward
// the ramp's value over `smoothFrames`.  With `settle`, a change at frame 0
// replaces the initial value.
template <class Transform>
Points automate(const Score& score, int cc, float initial, int smoothFrames, Transform transform, bool settle)
{
    struct Ramp {
        int first, last;
        float from, to;
    };
    float previous = transform(initial);
    Points points{{0, previous, 0}};
    std::vector<Ramp> ramps;
    int lastFrame = 0;
    for (const TimedEvent& e : score.events) {
        float value;
        if (e.type == EventType::control && e.data1 == 121) value = initial;
        else if (cc == 128 && e.type == EventType::bend) value = float(e.data1);
        else if (e.type == EventType::control && e.data1 == cc) value = float(e.data2);
        else continue;
        const float target = transform(value);
        if (settle && e.frame == 0)
            points.front().value = target;
        else if (target != previous)
            ramps.push_back({std::max(lastFrame, e.frame / kBendBlock * kBendBlock), e.frame, previous, target});
        previous = target;
        lastFrame = e.frame;
    }
    // Appends a point unless the track already passes through it with that slope.
    const auto put = [&points](int frame, float value, float step) {
        cs_control_point& back = points.back();
        if (back.frame == frame)
            back = {frame, value, step};
        else if (back.step != step || std::abs(back.value + (frame - back.frame) * step - value) > 1e-6f)
            points.push_back({frame, value, step});
    };
    if (smoothFrames < 2) {
        for (const Ramp& r : ramps) {
            if (r.first < r.last)
                put(r.first, r.from, (r.to - r.from) / (r.last - r.first));
            put(r.last, r.to, 0);
        }
        return points;
    }
    constexpr int kGroup = 16;
    const int smooth = std::max(kGroup, smoothFrames);
    float current = points.front().value, target = current, step = 0;
    size_t next = 0;
    for (int frame = 0; next < ramps.size() || current != target; frame += kGroup) {
        if (current == target && next < ramps.size() && frame < ramps[next].first)
            frame = std::max(frame, ramps[next].first / kGroup * kGroup);
        float aim = target;
        const int groupEnd = frame + kGroup - 1;
        while (next < ramps.size() && groupEnd >= ramps[next].last)
            aim = ramps[next++].to;
        if (next < ramps.size() && groupEnd >= ramps[next].first) {
            const Ramp& r = ramps[next];
            aim = r.from + (r.to - r.from) * (float(groupEnd - r.first) / (r.last - r.first));
        }
        if (aim != target) {
            target = aim;
            step = (target - current) / smooth;
        }
        if (current == target || step == 0) {
            put(frame, current, 0);
            continue;
        }
        put(frame, current + step, step);
        const float remaining = std::abs((target - current) / step);
        if (remaining <= kGroup) {
            put(frame + std::max(0, int(std::ceil(remaining)) - 1), target, 0);
            current = target;
        } else {
            current += kGroup * step;
        }
    }
    return points;
}

class TrackBook {
public:
    TrackBook(Plan& plan, const Score& score, const Instrument& instrument, int rate, bool natural)
        : plan_(plan), score_(score), instrument_(instrument), rate_(rate), natural_(natural) {}

    // The job's CC7 (volume), CC11 (expression) and CC10 (pan) tracks, as tracks
    // 0-2: constant when the instrument maps the controller itself.
    void addJobTracks()
    {
        for (const int cc : {7, 11, 10}) {
            if (instrument_.ccInUse[size_t(cc)]) {
                plan_.tracks.push_back({{0, cc == 10 ? 0.f : 1.f, 0}});
                continue;
            }
            const int curve = cc == 10 ? 1 : 4;
            plan_.tracks.push_back(automate(score_, cc, instrument_.startCc[size_t(cc)], rate_ / 100,
                                            [this, curve](float v) { return applyCurve(instrument_, curve, v); },
                                            natural_));
        }
    }

    int controller(const CcBinding& b)
    {
        return memo(controllers_, std::make_tuple(b.cc, b.curve, b.smoothMs), [&] {
            const int curve = b.curve;
            return automate(score_, b.cc, instrument_.startCc[size_t(b.cc)], b.smoothMs * rate_ / 1000,
                            [this, curve](float v) { return applyCurve(instrument_, curve, v); }, natural_);
        });
    }

    int smoothBend(const Pitch& p)
    {
        return memo(bends_, std::make_tuple(p.bendUp, p.bendDown, p.bendSmoothMs), [&] {
            const float up = p.bendUp, down = p.bendDown;
            return automate(score_, 128, 0, p.bendSmoothMs * rate_ / 1000, [up, down](float v) {
                const float bend = std::max(-8191.f, v) / 8191;
                return bend >= 0 ? bend * up : -bend * down;
            }, natural_);
        });
    }

    int ccFade(int cc, const Crossfade& xf)
    {
        return memo(fades_, std::make_tuple(cc, xf.inLo, xf.inHi, xf.outLo, xf.outHi, xf.power), [&] {
            return automate(score_, cc, instrument_.startCc[size_t(cc)], rate_ / 200,
                            [xf](float v) { return crossfade(xf, v, true); }, natural_);
        });
    }

    // A new empty track (LFO outputs, flex envelope shapes).
    int fresh()
    {
        plan_.tracks.emplace_back();
        return int(plan_.tracks.size()) - 1;
    }

    Points& operator[](int index) { return plan_.tracks[size_t(index)]; }

private:
    template <class Key, class Make>
    int memo(std::map<Key, int>& table, const Key& key, Make make)
    {
        const auto found = table.find(key);
        if (found != table.end())
            return found->second;
        const int index = int(plan_.tracks.size());
        table.emplace(key, index);
        plan_.tracks.push_back(make());
        return index;
    }

    Plan& plan_;
    const Score& score_;
    const Instrument& instrument_;
    int rate_;
    bool natural_;
    std::map<std::tuple<int, int, int>, int> controllers_;
    std::map<std::tuple<float, float, int>, int> bends_;
    std::map<std::tuple<int, int, int, int, int, bool>, int> fades_;
};

// ---- performance state and voices -------------------------------------------------------

enum class Cause { note, release, controller };     // what started a voice

// Controller and key state of the performance that parameter evaluation reads.
struct PlayState {
    std::array<float, 128> cc{};
    std::array<bool, 128> keyDown{};
    int keysDown = 0;
    float keyDelta = 0, noteRandom = 0;     // extended sources 140/141, 135/136
    bool alternate = false;                 // extended source 137
    std::mt19937 layers, variation;         // region layer draws; per-voice variation
    std::mt19937 noteDraws{1};              // the per-note random value

    PlayState(unsigned seed) : layers(seed), variation(seed ^ 0x85ebca6b) {}
};

struct BendSegment {
    int begin = 0, end = 0, from = 0, to = 0;
};

struct Voice {
    cs_voice_span span;
    int key, velocity, triggered;
    const Region* region;
    double baseStep;
    float releaseSeconds;
    bool keyReleased = false;
    Cause cause;
    bool choked = false, sostenuto = false;
    std::vector<int> flexTracks;        // pitch shapes cut at the voice's release
};

// The value of a binding's source for a voice (controllers, key, velocity and the
// extended sources), through the binding's curve.
float sourceValue(const Instrument& inst, const PlayState& state, const CcBinding& b, int key, int velocity,
                  Cause cause)
{
    if (b.cc == 140)
        return state.keyDelta;
    if (b.cc == 141)
        return std::abs(state.keyDelta);
    float value = 0;
    if (b.cc < 128) value = state.cc[size_t(b.cc)];
    else if (b.cc == 133) value = float(key);
    else if ((b.cc == 131 && cause == Cause::note) || (b.cc == 132 && cause == Cause::release)) value = float(velocity);
    else if (b.cc == 134) value = state.keysDown > 0 ? 127.f : 0.f;
    else if (b.cc == 135) value = 127 * state.noteRandom;
    else if (b.cc == 136) value = 127 * (2 * state.noteRandom - 1);
    else if (b.cc == 137) value = state.alternate ? 127.f : 0.f;
    else if (const auto found = inst.extendedDefaults.find(b.cc); found != inst.extendedDefaults.end())
        value = found->second;
    return applyCurve(inst, b.curve, value);
}

// A region parameter for a voice: `base` plus the amplitude envelope's velocity
// tracking (for its stages) plus every controller binding of the parameter.
float modulated(const Instrument& inst, const PlayState& state, const Region& r, int target, float base, int key,
                int velocity, Cause cause)
{
    if (target >= CS_MOD_ENV_DELAY && target <= CS_MOD_ENV_RELEASE)
        base += r.ampEnvelope.perVelocity[size_t(target - CS_MOD_ENV_DELAY)] * (velocity / 127.f);
    for (const CcBinding& b : r.bindings)
        if (b.target == target)
            base += b.depth * sourceValue(inst, state, b, key, velocity, cause);
    return base;
}

// The span's pitch at its begin frame under the current bend segment; regions
// with bend smoothing take the bend through a control track instead.
void bendSpan(Voice& v, const BendSegment& bend)
{
    cs_voice_span& span = v.span;
    const Pitch& pitch = v.region->pitch;
    if (pitch.bendSmoothMs > 0) {
        span.bendEnd = span.begin;
        span.pitchSlope = 0;
        span.step = v.baseStep;
        return;
    }
    const auto cents = [&pitch](int value) {
        const double normalized = std::max(-8191, value) / 8191.0;
        return normalized >= 0 ? normalized * pitch.bendUp : -normalized * pitch.bendDown;
    };
    const double to = cents(bend.to);
    span.bendEnd = bend.end;
    span.pitchSlope = 0;
    if (span.begin < bend.end) {
        const double from = cents(bend.from);
        const double slope = (to - from) / (bend.end - bend.begin);
        span.pitchSlope = slope * (std::log(2.) / 1200);
        span.step = v.baseStep * std::exp2((from + (span.begin - bend.begin) * slope) / 1200);
    } else {
        span.step = v.baseStep * std::exp2(to / 1200);
    }
}

// ---- LFOs ------------------------------------------------------------------------------------

class LfoBaker {
public:
    struct Lfo {
        const LfoSpec* spec;
        int begin, end, delay, fade;
        std::vector<cs_voice_modulation> inputs;     // first: track (or -1 for a constant depth)
        std::vector<std::pair<int, int>> outputs;    // (target, track)
    };

    // Registers the voice's LFOs (from `frame`): their controller inputs, and an
    // output track and binding per modulated target.  Returns the LFOs' pitch
    // depth bound; sets `stereo` when an LFO moves width or position.
    float add(Voice& v, int frame, bool& stereo, const Instrument& inst, const PlayState& state, TrackBook& tracks,
              Plan& plan, int rate)
    {
        cs_voice_span& span = v.span;
        span.firstLfo = int(lfos_.size());
        float pitchBound = 0;
        for (const auto& [index, spec] : v.region->lfos) {
            Lfo lfo{&spec, frame, frame, 0, 0, {}, {}};
            float delay = spec.delay, fade = spec.fade;
            Keyed<int, float> bound = spec.depth;
            for (auto& [target, depth] : bound)
                depth = std::abs(depth);
            for (const CcBinding& b : spec.ccs) {
                const float value = sourceValue(inst, state, b, v.key, v.velocity, v.cause);
                if (b.target == CS_MOD_LFO_DELAY) {
                    delay += b.depth * value;
                } else if (b.target == CS_MOD_LFO_FADE) {
                    fade += b.depth * value;
                } else {
                    const int track = b.cc < 128 ? tracks.controller(b) : -1;
                    lfo.inputs.push_back({track, 0, b.target, track < 0 ? b.depth * value : b.depth});
                    if (b.target < CS_MOD_LFO_FREQUENCY || b.target >= CS_MOD_EQ1_FREQUENCY) {
                        float maximum = std::abs(value);
                        if (track >= 0)
                            for (const cs_control_point& p : tracks[track])
                                maximum = std::max(maximum, std::abs(p.value));
                        bound.slot(b.target) += std::abs(b.depth) * maximum;
                    }
                }
            }
            lfo.delay = int(std::clamp(delay, 0.f, 100.f) * rate);
            lfo.fade = int(std::clamp(fade, 0.f, 100.f) * rate);
            for (const auto& [target, depth] : bound) {
                if (depth == 0)
                    continue;
                stereo |= target == CS_MOD_WIDTH || target == CS_MOD_POSITION;
                if (target == CS_MOD_PITCH)
                    pitchBound += depth;
                const int track = tracks.fresh();
                lfo.outputs.emplace_back(target, track);
                plan.bindings.push_back({track, 0, target, 1, -1, 0});
            }
            if (!lfo.outputs.empty())
                lfos_.push_back(std::move(lfo));
        }
        span.lfoCount = int(lfos_.size()) - span.firstLfo;
        return pitchBound;
    }

    // A span of the voice now ends at `end`: its LFOs run at least that long.
    void extend(const cs_voice_span& span)
    {
        for (int i = span.firstLfo; i < span.firstLfo + span.lfoCount; ++i)
            lfos_[size_t(i)].end = std::max(lfos_[size_t(i)].end, span.end);
    }

    // Output tracks of every LFO from its delayed start to its end: every 16
    // frames for the smooth waves (interpolated), every frame for the others.
    void bake(TrackBook& tracks, int rate)
    {
        std::mt19937 sampleHold(1);
        for (const Lfo& lfo : lfos_) {
            const LfoSpec& spec = *lfo.spec;
            const int start = lfo.begin + lfo.delay;
            const int stride = spec.wave <= 1 ? 16 : 1;
            double phase = 0;
            int cycle = -1;
            float held = 0;
            std::array<float, CS_MOD_EQ3_GAIN + 1> base{};
            for (const auto& [target, depth] : spec.depth)
                base[size_t(target)] = depth;
            for (const auto& [target, track] : lfo.outputs)
                tracks[track].push_back({0, 0, 0});
            for (int frame = start; frame < lfo.end; frame += stride) {
                float frequency = spec.frequency, shift = spec.phase;
                auto depth = base;
                for (const cs_voice_modulation& in : lfo.inputs) {
                    const float value = in.first < 0 ? in.depth : in.depth * valueAt(tracks[in.first], frame);
                    if (in.target == CS_MOD_LFO_FREQUENCY) frequency += value;
                    else if (in.target == CS_MOD_LFO_PHASE) shift += value;
                    else depth[size_t(in.target)] += value;
                }
                float wave = lfoShape(spec.wave, phase + shift);
                if (spec.wave == 12) {          // sample and hold: a new value each cycle
                    const int now = static_cast<int>(phase);
                    if (cycle != now) {
                        held = 2 * uniform24(sampleHold) - 1;
                        cycle = now;
                    }
                    wave = held;
                }
                const float fade = lfo.fade == 0 ? 1.f : std::min(1.f, float(frame - start) / lfo.fade);
                for (const auto& [target, track] : lfo.outputs) {
                    Points& points = tracks[track];
                    const float value = depth[size_t(target)] * wave * fade;
                    if (points.back().frame == frame) {
                        points.back().value = value;
                        continue;
                    }
                    if (stride > 1 && frame - points.back().frame == stride)
                        points.back().step = (value - points.back().value) / stride;
                    if (stride > 1 || value != points.back().value)
                        points.push_back({frame, value, 0});
                }
                phase += double(std::clamp(frequency, 0.f, 1000.f)) * stride / rate;
            }
        }
    }

private:
    std::vector<Lfo> lfos_;
};

cs_voice_modulation binding(int track, int target, float depth, int shape = -1)
{
    return cs_voice_modulation{track, 0, target, depth, shape, 0};
}

// ---- the performer ---------------------------------------------------------------------------

class Performer {
public:
    Performer(const Instrument& inst, SampleBank& bank, const Score& score, int rate, unsigned seed, int limit,
              TailPolicy tail)
        : inst_(inst), bank_(bank), score_(score), rate_(rate), limit_(limit), natural_(tail == TailPolicy::natural),
          state_(seed), roundRobin_(inst.regions.size(), 0u), keySwitch_(inst.startSwitch),
          tracks_(plan_, score, inst, rate, tail == TailPolicy::natural)
    {
        state_.cc = inst.startCc;
    }

    Plan play()
    {
        anyBend_ = std::any_of(score_.events.begin(), score_.events.end(),
                               [](const TimedEvent& e) { return e.type == EventType::bend && e.data1 != 0; });
        tracks_.addJobTracks();
        const std::vector<BendSegment> bends = bendSegments();
        size_t nextBend = 0;
        for (const TimedEvent& e : score_.events) {
            while (nextBend < bends.size() && bends[nextBend].begin <= e.frame)
                onBendSegment(bends[nextBend++]);
            retireEnded(e.frame);
            switch (e.type) {
            case EventType::noteOn: onNoteOn(e); break;
            case EventType::noteOff: onNoteOff(e); break;
            case EventType::control: onControl(e); break;
            case EventType::bend: break;
            }
        }
        retireEnded(score_.endFrame);
        for (Voice& v : sounding_) {
            // Natural renders end notes through the prepared MIDI and its pedals;
            // the other policies release what still holds at the end.
            if (!natural_ && v.cause == Cause::note && v.region->source.loop != LoopKind::oneShot)
                releaseVoice(v, score_.endFrame);
            if (v.span.end == kForever && limit_ == kForever)
                fail("a looping one-shot or release sample has no finite end");
            emit(v.span, v.span.end);
        }
        if (!natural_)
            plan_.frames = std::max(plan_.frames, score_.endFrame);
        if (plan_.spans.empty())
            fail("no playable notes for this SFZ and MIDI");
        lfos_.bake(tracks_, rate_);
        return std::move(plan_);
    }

private:
    const Instrument& inst_;
    SampleBank& bank_;
    const Score& score_;
    int rate_, limit_;
    bool natural_;
    PlayState state_;
    std::vector<unsigned> roundRobin_;          // per region: notes seen (sequence counters)
    int keySwitch_;
    int lastNote_ = -1, previousNote_ = -1;
    std::array<int, 128> noteStart_{}, noteVelocity_{};
    std::array<bool, 128> sostenutoKeys_{};
    bool sostenutoDown_ = false;
    bool anyBend_ = false;
    BendSegment bend_;
    struct Deferred {                           // a release layer waiting for a pedal
        int key, velocity, duration;
        const Region* region;
        bool sostenuto;
    };
    std::vector<Deferred> deferred_;
    std::vector<Voice> sounding_;
    Plan plan_;
    TrackBook tracks_;
    LfoBaker lfos_;

    // ---- spans -------------------------------------------------------------------

    // Emits the span, ending at `end` and at the render limit.
    void emit(cs_voice_span span, int end)
    {
        span.end = std::min(span.end, end);
        plan_.tailClipped |= span.end > limit_ && span.begin < span.end;
        span.end = std::min(span.end, limit_);
        if (span.begin >= span.end)
            return;
        lfos_.extend(span);
        plan_.frames = std::max(plan_.frames, span.end);
        plan_.spans.push_back(span);
    }

    // Voices whose span ended by `frame` are emitted and dropped.
    void retireEnded(int frame)
    {
        const auto kept = std::remove_if(sounding_.begin(), sounding_.end(), [&](const Voice& v) {
            if (v.span.end > frame)
                return false;
            emit(v.span, v.span.end);
            return true;
        });
        sounding_.erase(kept, sounding_.end());
    }

    // Ends the voice's current span at `frame`; the voice continues in a new span
    // from source position `position`.
    void cutSpan(Voice& v, int frame, double position)
    {
        emit(v.span, frame);
        v.span.begin = frame;
        v.span.position = position;
    }

    int envelopeEnd(const cs_voice_span& span) const
    {
        return span.releaseStart < 0 ? kForever : span.fadeStart + rate_ / 20 + 1;
    }

    // ---- pitch bend --------------------------------------------------------------------

    // Bend changes as segments: a ramp from the change's 1024-frame block to the
    // event (the format's block interpolation), then the held value.
    std::vector<BendSegment> bendSegments() const
    {
        std::vector<BendSegment> out;
        int lastFrame = 0, lastValue = 0;
        for (const TimedEvent& e : score_.events) {
            const bool reset = e.type == EventType::control && e.data1 == 121;
            if (e.type != EventType::bend && !reset)
                continue;
            const int value = reset ? 0 : e.data1;
            const int begin = std::max(lastFrame, e.frame / kBendBlock * kBendBlock);
            if (lastValue != value) {
                out.push_back({begin, e.frame, lastValue, value});
                out.push_back({e.frame, e.frame, value, value});
            }
            lastFrame = e.frame;
            lastValue = value;
        }
        return out;
    }

    void onBendSegment(const BendSegment& segment)
    {
        retireEnded(segment.begin);
        bend_ = segment;
        for (Voice& v : sounding_) {
            if (v.region->pitch.bendSmoothMs > 0)
                continue;
            const int at = std::max(segment.begin, v.span.begin);
            cutSpan(v, at, v.span.position + travelled(v.span, at - v.span.begin));
            bendSpan(v, bend_);
            v.span.end = spanEnd(v.span, envelopeEnd(v.span));
        }
    }

    // ---- starting a voice ----------------------------------------------------------------

    float param(const Region& r, int target, float base, int key, int velocity, Cause cause) const
    {
        return modulated(inst_, state_, r, target, base, key, velocity, cause);
    }

    float variation(float extent) { return extent == 0 ? 0.f : extent * uniform24(state_.variation); }

    // Starts a voice of region `r` for `key` at `frame`: choke groups and per-note
    // polyphony first, then the span (see buildSpan).  `held` is the note's held
    // frames (release layers), `ccSource` the controller of a CC trigger.
    void startVoice(const Region& r, int frame, int key, int velocity, Cause cause, int held = 0, int ccSource = -1)
    {
        if (inst_.anyChoke)
            chokeGroups(r, frame, ccSource >= 0 ? ccSource : key, cause);
        if (r.rules.notePolyphony)
            capNoteVoices(r, frame, key, velocity);
        Voice v{};
        v.key = key;
        v.velocity = velocity;
        v.triggered = frame;
        v.region = &r;
        v.cause = cause;
        buildSpan(v, frame, held);
        sounding_.push_back(std::move(v));
    }

    void buildSpan(Voice& v, int frame, int held)
    {
        const Region& r = *v.region;
        const int key = v.key, velocity = v.velocity;
        const Cause cause = v.cause;
        const Sample* sample = r.source.generator == CS_GEN_NONE ? &bank_.decode(r.source.sampleId) : nullptr;
        const auto at = [&](int target, float base) { return param(r, target, base, key, velocity, cause); };
        const auto seconds = [&](int target, float base) { return std::clamp(at(target, base), 0.f, 100.f); };
        const auto& amp = r.ampEnvelope.stage;
        cs_voice_span& span = v.span;

        // Source and pitch.
        v.releaseSeconds = seconds(CS_MOD_ENV_RELEASE, amp[kRelease]);
        const double sourceRate = sample ? sample->rate : 440 * std::exp2((r.select.center - 69) / 12.);
        v.baseStep = (sourceRate / rate_) *
            std::exp2((r.pitch.keyTrack * (key - r.select.center) + r.pitch.tune + 100 * r.pitch.transpose +
                       variation(r.pitch.random)) / 1200.0);
        span.sample = sample ? sample->offset : 0;
        span.channels = sample ? sample->channels : 1;
        span.generator = r.source.generator;
        if (r.source.generator == CS_GEN_NOISE) {
            span.noiseSeed = state_.variation();
            span.noiseStart = frame;
        }
        span.begin = frame + int(seconds(CS_MOD_DELAY, r.rules.delay) * rate_);
        span.sourceEnd = r.source.end;
        const int offsetJitter = r.source.offsetRandom
            ? std::uniform_int_distribution<int>(0, r.source.offsetRandom)(state_.variation) : 0;
        if (sample) {
            span.position = std::trunc(std::clamp(double(at(CS_MOD_OFFSET, float(r.source.offset))) + offsetJitter, 0.,
                                                  double(r.source.end)));
        } else {
            const float phase = r.source.oscillatorPhase >= 0 ? r.source.oscillatorPhase : state_.noteRandom;
            span.position = phase - std::floor(phase);
        }
        bendSpan(v, bend_);
        if (sample && (r.source.loop == LoopKind::continuous || r.source.loop == LoopKind::sustain)) {
            span.loopFirst = r.source.loopStart;
            span.loopEnd = r.source.loopEnd;
            span.loopCrossfade = static_cast<int>(
                std::lround(std::min<double>(r.source.loopStart, double(r.source.loopCrossfade) * sample->rate)));
        }

        // Amplitude envelope.
        span.start = std::clamp(at(CS_MOD_ENV_START, amp[kStart]), 0.f, 1.f);
        span.attackStart = span.begin + int(seconds(CS_MOD_ENV_DELAY, amp[kDelay]) * rate_);
        const float attackFrames = seconds(CS_MOD_ENV_ATTACK, amp[kAttack]) * rate_;
        span.attackStep = attackFrames > 0 ? 1 / attackFrames : 1;
        span.holdStart = span.attackStart + std::max(0, int(std::ceil((1 - span.start) * attackFrames)) - 1);
        span.decayStart = span.holdStart + int(seconds(CS_MOD_ENV_HOLD, amp[kHold]) * rate_);
        const float decay = seconds(CS_MOD_ENV_DECAY, amp[kDecay]);
        span.decayRate = decay > 0 ? -9 / (std::max(.006f, decay) * rate_) : 0;
        span.sustain = std::clamp(at(CS_MOD_ENV_SUSTAIN, amp[kSustain]), 0.f, 1.f);
        span.releaseStart = -1;
        auxShapes(v);

        // Filters and EQ bands, sharing the voice's filter chain.
        span.filterTrack = -1;
        span.sampleRate = rate_;
        for (size_t i = 0; i < r.filters.size(); ++i) {
            const FilterSpec& f = r.filters[i];
            if (f.type == CS_FILTER_NONE)
                continue;
            if (span.filterTrack < 0)
                span.filterTrack = plan_.filterTracks++;
            const int velocityTarget = i == 0 ? CS_MOD_FILTER_VELOCITY : CS_MOD_FILTER_VELOCITY2;
            const float cents = f.keyTrack * (key - f.keyCenter) + variation(f.random) +
                at(velocityTarget, f.velocityTrack) * velocity / 127.f;
            span.filters[i] = {f.type,
                               std::clamp(f.cutoff * std::exp2(std::clamp(cents, -24000.f, 24000.f) / 1200), 0.f, 20000.f),
                               f.resonance, 0, 0};
        }
        static constexpr float kEqCentre[] = {50, 500, 5000};
        for (size_t i = 0; i < r.eqs.size(); ++i) {
            const EqSpec& eq = r.eqs[i];
            if (!eq.on)
                continue;
            if (span.filterTrack < 0)
                span.filterTrack = plan_.filterTracks++;
            span.filters[i + 2] = {CS_FILTER_PEAK, eq.frequency == 0 ? kEqCentre[i] : eq.frequency, 0, eq.bandwidth,
                                   eq.gain};
        }

        // Modulation bindings, LFOs and pitch shapes; the pitch bound decides
        // whether the phase is integrated per frame.
        span.firstModulation = int(plan_.bindings.size());
        bool stereoModulated = false;
        float pitchBound = std::abs(span.extraEnvelope[1].depth);
        for (const CcBinding& b : r.bindings) {
            if ((b.target >= CS_MOD_ENV_DELAY && b.target < CS_MOD_CUTOFF) ||
                (b.target >= CS_MOD_FILTER_VELOCITY && b.target < CS_MOD_FILEG_DEPTH))
                continue;               // start-time parameters, already applied
            stereoModulated |= b.target == CS_MOD_WIDTH || b.target == CS_MOD_POSITION;
            if (b.target == CS_MOD_PITCH || b.target == CS_MOD_PITCHEG_DEPTH)
                pitchBound += std::abs(b.cc < 128 ? b.depth : b.depth * sourceValue(inst_, state_, b, key, velocity, cause));
            if (b.cc < 128)
                plan_.bindings.push_back(binding(tracks_.controller(b), b.target, b.depth));
            else
                plan_.bindings.push_back(binding(-1, b.target, b.depth * sourceValue(inst_, state_, b, key, velocity, cause)));
        }
        for (const auto& [cc, xf] : r.amp.ccFades)
            plan_.bindings.push_back(binding(tracks_.ccFade(cc, xf), CS_MOD_AMPLITUDE, 1));
        if (r.pitch.bendSmoothMs > 0 && anyBend_) {
            pitchBound += std::max(std::abs(r.pitch.bendUp), std::abs(r.pitch.bendDown));
            plan_.bindings.push_back(binding(tracks_.smoothBend(r.pitch), CS_MOD_PITCH, 1));
        }
        pitchBound += lfos_.add(v, frame, stereoModulated, inst_, state_, tracks_, plan_, rate_);
        pitchBound += flexShapes(v);
        span.minimumPitchRatio = std::exp2(-std::min(24000.f, pitchBound) / 1200);
        if (pitchBound > 0) {
            span.variablePitch = 1;
            if (span.filterTrack < 0)
                span.filterTrack = plan_.filterTracks++;
        }
        span.modulationCount = int(plan_.bindings.size()) - span.firstModulation;

        // Gains and stereo placement.
        const float noteGain = cause == Cause::controller ? 1.f
            : velocityGain(r, velocity) * crossfade(r.amp.keyFade, key, false) * crossfade(r.amp.velocityFade, velocity, true);
        const float gain = r.amp.linear * noteGain *
            std::pow(10.f, ((natural_ ? 0 : kMasterDb) + r.amp.volumeDb + variation(r.amp.randomDb) -
                            r.rules.releaseDecay * held / rate_ + 3) / 20);
        constexpr float kQuarterPi = .7853981633974483f;
        constexpr float kPanCompensation = 1.4125375446227544f;
        const bool matrix = span.channels == 2 && (stereoModulated || r.amp.width != 1 || r.amp.position != 0);
        span.stereoMatrix = matrix;
        span.gain = gain * (matrix ? kPanCompensation : span.channels == 1 ? 1.f : .99881488f);
        span.pan = r.amp.pan;
        span.width = r.amp.width;
        span.stereoPosition = r.amp.position;
        span.left = span.gain * std::cos((1 + r.amp.pan) * kQuarterPi);
        span.right = span.gain * std::cos((1 - r.amp.pan) * kQuarterPi);
        span.widthDirect = matrix ? std::cos((1 - r.amp.width) * kQuarterPi) : 1.f;
        span.widthCross = matrix ? std::cos((1 + r.amp.width) * kQuarterPi) : 0.f;
        span.positionLeft = matrix ? std::cos((1 + r.amp.position) * kQuarterPi) : 1.f;
        span.positionRight = matrix ? std::cos((1 - r.amp.position) * kQuarterPi) : 1.f;
        span.end = spanEnd(span, kForever);
    }

    // The filter (slot 0) and pitch (slot 1) envelopes of the voice.
    void auxShapes(Voice& v)
    {
        cs_voice_span& span = v.span;
        const Region& r = *v.region;
        for (int slot = 0; slot < 2; ++slot) {
            const AuxEnvelope& env = r.aux[size_t(slot)];
            if (!env.on)
                continue;
            const int first = slot == 0 ? CS_MOD_FILEG_DELAY : CS_MOD_PITCHEG_DELAY;
            std::array<float, kStages> stage;
            for (int p = 0; p < kStages; ++p) {
                const float base = env.shape.stage[size_t(p)] + env.shape.perVelocity[size_t(p)] * (v.velocity / 127.f);
                const float value = param(r, first + p, base, v.key, v.velocity, v.cause);
                stage[size_t(p)] = std::clamp(value, 0.f, p == kSustain || p == kStart ? 1.f : 100.f);
            }
            cs_envelope_shape& shape = span.extraEnvelope[slot];
            span.activeEnvelope[slot] = 1;
            shape.start = stage[kStart];
            shape.attackStart = span.begin + int(stage[kDelay] * rate_);
            const float attack = stage[kAttack] * rate_;
            shape.attackStep = attack > 0 ? 1 / attack : 1;
            shape.holdStart = shape.attackStart + std::max(0, int(std::ceil((1 - shape.start) * attack)) - 1);
            shape.decayStart = shape.holdStart + int(stage[kHold] * rate_);
            shape.decayRate = stage[kDecay] > 0 ? -9 / (std::max(.006f, stage[kDecay]) * rate_) : 0;
            shape.sustain = stage[kSustain];
            shape.releaseStart = -1;
            shape.releaseSeconds = stage[kRelease];
            shape.depth = env.depth + env.velocityDepth * (v.velocity / 127.f);
        }
    }

    // Flex envelopes on pitch: a shape track per envelope from the voice's trigger
    // (stage times may follow controllers), bound to pitch with its depths.
    float flexShapes(Voice& v)
    {
        float bound = 0;
        for (const auto& [id, env] : v.region->flex) {
            std::vector<cs_voice_modulation> depths;
            if (env.pitch != 0) {
                depths.push_back(binding(-1, CS_MOD_PITCH, env.pitch));
                bound += std::abs(env.pitch);
            }
            for (const auto& [cc, depth] : env.pitchCc) {
                const CcBinding source{CS_MOD_PITCH, cc, depth};
                const float value = sourceValue(inst_, state_, source, v.key, v.velocity, v.cause);
                if (cc < 128) {
                    depths.push_back(binding(tracks_.controller(source), CS_MOD_PITCH, depth));
                    bound += std::abs(depth);
                } else if (value != 0) {
                    depths.push_back(binding(-1, CS_MOD_PITCH, depth * value));
                    bound += std::abs(depth * value);
                }
            }
            if (depths.empty())
                continue;
            const int shape = tracks_.fresh();
            v.flexTracks.push_back(shape);
            tracks_[shape].push_back({0, 0, 0});
            const auto put = [&](int frame, float level, float step) {
                Points& track = tracks_[shape];
                if (track.back().frame == frame)
                    track.back() = {frame, level, step};
                else
                    track.push_back({frame, level, step});
            };
            int frame = v.triggered;
            float level = 0;
            for (const auto& [index, stage] : env.stages) {
                float time = stage.seconds;
                for (const auto& [cc, perCc] : stage.secondsCc)
                    time += perCc * sourceValue(inst_, state_, CcBinding{CS_MOD_PITCH, cc}, v.key, v.velocity, v.cause);
                const int frames = int(std::clamp(time, 0.f, 100.f) * rate_);
                if (frames > 0)
                    put(frame, level, (stage.level - level) / frames);
                level = stage.level;
                frame += frames;
                put(frame, level, 0);
            }
            for (cs_voice_modulation m : depths) {
                m.shapeFirst = shape;
                plan_.bindings.push_back(m);
            }
        }
        return bound;
    }

    // ---- ending voices --------------------------------------------------------------------

    // A key's release: note voices that are not one-shots start their release
    // (re-reading a dynamic release time).
    void releaseVoice(Voice& v, int frame)
    {
        if (v.span.releaseStart >= 0 || v.cause != Cause::note || v.region->source.loop == LoopKind::oneShot)
            return;
        if (v.region->ampEnvelope.dynamic)
            v.releaseSeconds = param(*v.region, CS_MOD_ENV_RELEASE, v.region->ampEnvelope.stage[kRelease], v.key,
                                     v.velocity, v.cause);
        fadeOut(v, frame, v.releaseSeconds);
    }

    // Starts (or restarts) the release of the voice at `frame` over `seconds`: a
    // sustain loop is left, flex shapes return to zero, the filter and pitch
    // envelopes release too.
    void fadeOut(Voice& v, int frame, float seconds)
    {
        cs_voice_span& span = v.span;
        if (frame >= span.end)
            return;
        if (frame < span.begin) {
            span.end = span.begin;
            return;
        }
        const float level = levelAt(span, frame - 1);
        const bool leaveLoop = v.region->source.loop == LoopKind::sustain && span.loopEnd > 0;
        if (leaveLoop || span.releaseStart >= 0) {
            const double position = span.position + travelled(span, frame - span.begin);
            cutSpan(v, frame, leaveLoop ? wrapped(span, position) : position);
            bendSpan(v, bend_);
            if (leaveLoop)
                span.loopEnd = 0;
        }
        startReleaseCurve(span, frame, rate_, level, seconds);
        for (const int shape : v.flexTracks) {
            Points& track = tracks_[shape];
            track.erase(std::lower_bound(track.begin(), track.end(), frame,
                                         [](const cs_control_point& p, int f) { return p.frame < f; }),
                        track.end());
            track.push_back({frame, 0, 0});
        }
        for (int slot = 0; slot < 2; ++slot) {
            cs_envelope_shape& shape = span.extraEnvelope[slot];
            if (span.activeEnvelope[slot] && shape.releaseStart < 0)
                startReleaseCurve(shape, frame, rate_, levelAt(shape, frame - 1), shape.releaseSeconds);
        }
        span.end = spanEnd(span, envelopeEnd(span));
    }

    // A voice cut by its choke group or by polyphony, with its off mode's time.
    void cutVoice(Voice& v, int frame)
    {
        const VoiceRules& rules = v.region->rules;
        v.choked = true;
        const float time = rules.offMode == OffKind::normal ? v.releaseSeconds
            : rules.offMode == OffKind::fast ? .006f : rules.offTime;
        fadeOut(v, frame, time);
    }

    // Voices whose off_by names the incoming region's group are cut (not the
    // incoming note's own voices of the same group); cut note voices fire their
    // release layers.
    void chokeGroups(const Region& incoming, int frame, int key, Cause cause)
    {
        std::vector<std::pair<int, int>> notes;
        for (Voice& v : sounding_) {
            const Region& r = *v.region;
            if (v.span.end <= frame || v.cause == Cause::release || v.choked || !r.rules.chokedByGroup ||
                r.rules.offBy != incoming.rules.group ||
                (r.rules.group == incoming.rules.group && v.key == key && ccConditionsHold(r)))
                continue;
            cutVoice(v, frame);
            if (cause != Cause::controller && v.cause == Cause::note)
                notes.emplace_back(v.key, v.velocity);
        }
        for (const auto& [k, velocity] : notes)
            fireReleaseLayers(frame, k, velocity, std::max(0, frame - noteStart_[size_t(k)]));
    }

    // note_polyphony: at most that many voices of the region's group on the key;
    // the oldest (or, with self-masking, the quietest no louder than the new note)
    // are cut together with their sister voices of the same note.
    void capNoteVoices(const Region& region, int frame, int key, int velocity)
    {
        std::vector<Voice*> candidates;
        int count = 0;
        for (Voice& v : sounding_) {
            if (v.choked || v.span.end <= frame || v.key != key || v.region->rules.group != region.rules.group)
                continue;
            ++count;
            if (!region.rules.selfMask || v.velocity <= velocity)
                candidates.push_back(&v);
        }
        if (count < region.rules.notePolyphony)
            return;
        std::stable_sort(candidates.begin(), candidates.end(), [&](const Voice* a, const Voice* b) {
            return region.rules.selfMask ? a->velocity < b->velocity : a->triggered < b->triggered;
        });
        for (Voice* c : candidates) {
            if (c->choked)
                continue;
            for (Voice& sister : sounding_)
                if (!sister.choked && sister.key == c->key && sister.cause == c->cause && sister.triggered == c->triggered)
                    cutVoice(sister, frame);
            if (--count < region.rules.notePolyphony)
                break;
        }
    }

    // ---- selection ------------------------------------------------------------------------

    bool pedalDown(const Region& r) const
    {
        return r.rules.pedal && state_.cc[size_t(r.rules.pedalCc)] >= r.rules.pedalLow;
    }

    bool ccConditionsHold(const Region& r) const
    {
        return std::all_of(r.select.ccConditions.begin(), r.select.ccConditions.end(), [&](const CcRange& c) {
            return state_.cc[c.cc] >= c.lo && state_.cc[c.cc] <= c.hi;
        });
    }

    bool switchesHold(const Region& r) const
    {
        const Selection& s = r.select;
        return (s.switchLo < 0 || (keySwitch_ >= s.switchLo && keySwitch_ <= s.switchHi)) &&
            (s.switchDown < 0 || state_.keyDown[size_t(s.switchDown)]) &&
            (s.switchUp < 0 || !state_.keyDown[size_t(s.switchUp)]) &&
            (s.switchPrevious < 0 || previousNote_ == s.switchPrevious);
    }

    bool selected(const Region& r, int velocity, float draw) const
    {
        return r.select.velocities.contains(velocity) && draw >= r.select.randomLo && draw < r.select.randomHi &&
            switchesHold(r) && ccConditionsHold(r);
    }

    // Does a note voice sound within the region's key and velocity ranges?
    bool noteSounding(const Region& r) const
    {
        return std::any_of(sounding_.begin(), sounding_.end(), [&](const Voice& v) {
            return v.cause == Cause::note && r.select.keys.contains(v.key) && r.select.velocities.contains(v.velocity);
        });
    }

    // ---- events ------------------------------------------------------------------------------

    void onNoteOn(const TimedEvent& e)
    {
        const int key = e.data1, velocity = e.data2;
        const bool keySwitch = inst_.switchKey[size_t(key)];
        if (keySwitch)
            keySwitch_ = key;
        if (!state_.keyDown[size_t(key)] && !keySwitch)
            ++state_.keysDown;
        if (!keySwitch) {
            state_.keyDelta = lastNote_ < 0 ? 0.f : float(key - lastNote_);
            lastNote_ = key;
            state_.noteRandom = uniform24(state_.noteDraws);
            state_.alternate = !state_.alternate;
        }
        state_.keyDown[size_t(key)] = true;
        noteVelocity_[size_t(key)] = velocity;
        noteStart_[size_t(key)] = e.frame;
        const float draw = uniform24(state_.layers);
        for (const int index : inst_.regionsByKey[size_t(key)]) {
            const Region& r = inst_.regions[size_t(index)];
            const bool inTurn = roundRobin_[size_t(index)]++ % unsigned(r.select.sequenceLength) ==
                unsigned(r.select.sequencePosition - 1);
            if (!inTurn || !selected(r, velocity, draw))
                continue;
            const Trigger t = r.select.trigger;
            if (t == Trigger::attack || (t == Trigger::first && state_.keysDown == 1) ||
                (t == Trigger::legato && state_.keysDown > 1))
                startVoice(r, e.frame, key, velocity, Cause::note);
        }
        previousNote_ = key;
    }

    void onNoteOff(const TimedEvent& e)
    {
        const int key = e.data1;
        if (!state_.keyDown[size_t(key)])
            return;
        state_.keyDown[size_t(key)] = false;
        if (!inst_.switchKey[size_t(key)])
            --state_.keysDown;
        for (Voice& v : sounding_) {
            if (v.key != key || v.cause != Cause::note)
                continue;
            v.keyReleased = true;
            if (!pedalDown(*v.region) && !v.sostenuto)
                releaseVoice(v, e.frame);
        }
        fireReleaseLayers(e.frame, key, noteVelocity_[size_t(key)], e.frame - noteStart_[size_t(key)]);
    }

    // Release-triggered regions of `key`: sounded now, or deferred while a pedal
    // (or sostenuto) holds the note.
    void fireReleaseLayers(int frame, int key, int velocity, int held)
    {
        const float draw = uniform24(state_.layers);
        for (const int index : inst_.regionsByKey[size_t(key)]) {
            const Region& r = inst_.regions[size_t(index)];
            const unsigned seen = roundRobin_[size_t(index)];
            const bool inTurn = seen == 0 ? !r.select.sequenceExplicit
                                          : (seen - 1) % unsigned(r.select.sequenceLength) ==
                                                unsigned(r.select.sequencePosition - 1);
            const Trigger t = r.select.trigger;
            if ((t != Trigger::release && t != Trigger::releaseKey) || !inTurn || !selected(r, velocity, draw))
                continue;
            if (t == Trigger::release && (pedalDown(r) || sostenutoKeys_[size_t(key)]))
                deferred_.push_back({key, velocity, held, &r, sostenutoKeys_[size_t(key)]});
            else if (t == Trigger::releaseKey || r.rules.releaseDead || noteSounding(r))
                startVoice(r, frame, key, velocity, Cause::release, held);
        }
    }

    // A controller change may retune the release of voices with a dynamic
    // amplitude envelope (other mid-voice envelope changes are refused).
    void retuneEnvelopes(const std::array<float, 128>& before, int frame)
    {
        for (Voice& v : sounding_) {
            if (v.choked)
                continue;
            const Region& r = *v.region;
            for (const CcBinding& b : r.bindings) {
                if (b.cc >= 128 || before[size_t(b.cc)] == state_.cc[size_t(b.cc)] || b.depth == 0)
                    continue;
                const bool filterEg = b.target >= CS_MOD_FILEG_DELAY && b.target <= CS_MOD_FILEG_RELEASE;
                const bool pitchEg = b.target >= CS_MOD_PITCHEG_DELAY && b.target <= CS_MOD_PITCHEG_RELEASE;
                if ((filterEg && r.aux[0].shape.dynamic) || (pitchEg && r.aux[1].shape.dynamic))
                    fail("changing a dynamic pitch or filter envelope mid-voice is unsupported");
                if (!r.ampEnvelope.dynamic || b.target < CS_MOD_ENV_DELAY || b.target > CS_MOD_ENV_RELEASE)
                    continue;
                if (b.target != CS_MOD_ENV_RELEASE)
                    fail("changing a dynamic amplitude envelope mid-voice is unsupported for CC" + std::to_string(b.cc));
                if (v.span.releaseStart >= 0 && frame < v.span.fadeStart) {
                    fadeOut(v, frame, param(r, CS_MOD_ENV_RELEASE, r.ampEnvelope.stage[kRelease], v.key, v.velocity,
                                            v.cause));
                    break;
                }
            }
        }
    }

    void onControl(const TimedEvent& e)
    {
        const int cc = e.data1, value = e.data2;
        if (cc == 121) {                        // reset all controllers
            const auto before = state_.cc;
            state_.cc = inst_.startCc;
            retuneEnvelopes(before, e.frame);
            if (natural_) {
                setSostenuto(false);
                releasePedalled(e.frame, 66, before[66]);
            }
            for (Voice& v : sounding_)
                if (v.keyReleased && !pedalDown(*v.region))
                    releaseVoice(v, e.frame);
            return;
        }
        if (!natural_ && cc == 66 && value != 0)
            fail("unsupported MIDI sostenuto CC66");
        if (natural_ && (cc == 120 || cc == 123)) {     // all sound / notes off
            for (Voice& v : sounding_)
                emit(v.span, e.frame);
            sounding_.clear();
            deferred_.clear();
            state_.keyDown.fill(false);
            sostenutoKeys_.fill(false);
            state_.keysDown = 0;
            return;
        }
        if (cc >= 120)
            fail("unsupported MIDI channel mode CC" + std::to_string(cc));
        const bool sostenuto = natural_ && cc == 66;
        if (!inst_.ccInUse[size_t(cc)] && !sostenuto)
            return;
        const auto before = state_.cc;
        const float previous = before[size_t(cc)];
        state_.cc[size_t(cc)] = static_cast<float>(value);
        if (previous != state_.cc[size_t(cc)])
            retuneEnvelopes(before, e.frame);
        if (sostenuto)
            setSostenuto(value == 127);
        releasePedalled(e.frame, cc, previous);
        const auto& triggered = inst_.regionsByCc[size_t(cc)];
        if (triggered.empty())
            return;
        const float draw = uniform24(state_.layers);
        for (const int index : triggered) {
            const Region& r = inst_.regions[size_t(index)];
            const auto range = std::find_if(r.select.ccTriggers.begin(), r.select.ccTriggers.end(),
                                            [&](const CcRange& c) { return c.cc == cc; });
            if (value < range->lo || value > range->hi || draw < r.select.randomLo || draw >= r.select.randomHi)
                continue;
            const bool inTurn = roundRobin_[size_t(index)]++ % unsigned(r.select.sequenceLength) ==
                unsigned(r.select.sequencePosition - 1);
            if (inTurn && switchesHold(r) && previous != value && ccConditionsHold(r))
                startVoice(r, e.frame, r.select.center, value, Cause::controller, 0, cc);
        }
    }

    void setSostenuto(bool down)
    {
        if (sostenutoDown_ == down)
            return;
        sostenutoDown_ = down;
        sostenutoKeys_ = down ? state_.keyDown : std::array<bool, 128>{};
        for (Voice& v : sounding_)
            v.sostenuto = down && !v.keyReleased;
        if (!down)
            for (Deferred& d : deferred_)
                d.sostenuto = false;
    }

    // After a pedal controller changes: released keys no longer held sound their
    // release, and deferred release layers whose pedal lifted start.
    void releasePedalled(int frame, int cc, float previous)
    {
        const bool sostenutoLifted = natural_ && cc == 66 && !sostenutoDown_;
        for (Voice& v : sounding_) {
            const Region& r = *v.region;
            const bool pedalChanged = r.rules.pedal && r.rules.pedalCc == cc && previous >= r.rules.pedalLow;
            if (v.keyReleased && (pedalChanged || sostenutoLifted) && !pedalDown(r) && !v.sostenuto)
                releaseVoice(v, frame);
        }
        std::vector<Deferred> due;
        const auto kept = std::remove_if(deferred_.begin(), deferred_.end(), [&](const Deferred& d) {
            const Region& r = *d.region;
            if ((r.rules.pedalCc != cc && !sostenutoLifted) || pedalDown(r) || d.sostenuto)
                return false;
            if (r.rules.releaseDead || noteSounding(r))
                due.push_back(d);
            return true;
        });
        deferred_.erase(kept, deferred_.end());
        for (const Deferred& d : due)
            startVoice(*d.region, frame, d.key, d.velocity, Cause::release, d.duration);
    }
};

} // namespace

Plan planJob(const Instrument& instrument, SampleBank& bank, const Score& score, int rate, unsigned seed, int limit,
             TailPolicy tail)
{
    return Performer(instrument, bank, score, rate, seed, limit, tail).play();
}

} // namespace clayhost
