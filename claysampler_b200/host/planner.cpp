// The planner: a job's MIDI events against an instrument become voice spans,
// piecewise-linear control tracks and modulation bindings (the render path's
// input).  It restates the reference's src/render/plan.cpp step for step —
// triggers, release and pedal handling, choke groups, note polyphony, bends,
// LFO and envelope tracks, and every random draw in the same order — because
// event scheduling, region and layer selection, voice stealing, positions and
// lengths must match the reference bit for bit.
#include "host_types.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <random>
#include <stdexcept>
#include <tuple>

namespace csh {
namespace {

constexpr int forever = std::numeric_limits<int>::max();
constexpr float silence = 1e-4f;                    // release end: -80 dB (plan.cpp:15)
constexpr int referenceBlock = 1024;
constexpr float masterGainDb = -7.35f;
constexpr float quarterPi = .7853981633974483f;
constexpr float panCompensation = 1.4125375446227544f;

enum class VoiceKind { attack, release, controller };

struct Voice {
    cs_voice_span span;
    int key, velocity, triggerFrame;
    const Region* region;
    double baseStep;
    float releaseSeconds;
    bool noteOff = false;
    VoiceKind kind;
    bool choked = false, sostenuto = false;
    std::vector<int> flexShapes;
};

struct DelayedRelease {
    int key, velocity, duration;
    const Region* region;
    bool sostenuto;
};

struct Bend {
    int begin = 0, end = 0, from = 0, to = 0;
};

struct LfoTrack {
    const Lfo* source;
    int begin, end, delay, fade;
    std::vector<cs_voice_modulation> inputs;
    std::vector<std::pair<int, int>> outputs;       // target, track
};

using Track = std::vector<cs_control_point>;

float valueAt(const Track& track, int frame)
{
    const auto last = std::upper_bound(track.begin(), track.end(), frame,
        [](int value, const cs_control_point& point) { return value < point.frame; });
    const auto& point = last == track.begin() ? track.front() : *std::prev(last);
    return point.value + float(frame - point.frame) * point.step;
}

float lfoShape(int wave, double phase)
{
    const float p = static_cast<float>(phase - std::floor(phase));
    switch (wave) {
    case 0: return p < .25f ? 4 * p : p > .75f ? 4 * p - 4 : 2 - 4 * p;
    case 1: {
        const float x = 2 * p - 1;
        return -4 * x * (1 - std::abs(x));
    }
    case 2: return p < .75f;
    case 3: return p < .5f;
    case 4: return p < .25f;
    case 5: return p < .125f;
    case 6: return 2 * p - 1;
    case 7: return 1 - 2 * p;
    default: return 0;
    }
}

float velocityGain(const Region& r, int velocity)
{
    const float normalized = float(velocity) / 127;
    float gain = normalized * normalized;
    if (!r.velocityCurve.empty()) {
        const auto last = std::lower_bound(r.velocityCurve.begin(), r.velocityCurve.end(), velocity,
                                           [](const auto& point, int value) { return point.first < value; });
        if (last->first == velocity) {
            gain = last->second;
        } else {
            const auto first = std::prev(last);
            const float phase = float(velocity - first->first) / float(last->first - first->first);
            gain = first->second + phase * (last->second - first->second);
        }
    }
    const float track = std::abs(r.velocityTrack) * (1 - gain);
    return r.velocityTrack < 0 ? track : 1 - track;
}

float crossfadeGain(const Crossfade& fade, float value, bool controllerScale)
{
    const auto top = [controllerScale](int high) { return controllerScale && high == 127 ? 126 : high; };
    const int inHigh = top(fade.inHigh), outHigh = top(fade.outHigh);
    float up = 1, down = 1;
    if (value < fade.inLow)
        up = 0;
    else if (inHigh > fade.inLow)
        up = std::min(1.f, float(value - fade.inLow) / float(inHigh - fade.inLow));
    if (outHigh > fade.outLow)
        down = std::clamp(float(outHigh - value) / float(outHigh - fade.outLow), 0.f, 1.f);
    return fade.power ? std::sqrt(up * down) : up * down;
}

// Pitch-bend ramps, interpolated within the 1024-frame block as sfizz does.
std::vector<Bend> bendRamps(const Midi& midi)
{
    std::vector<Bend> bends;
    int previousFrame = 0, previousValue = 0;
    for (const auto& event : midi.events) {
        const bool reset = event.kind == EventKind::control && event.a == 121;
        if (event.kind != EventKind::bend && !reset)
            continue;
        const int value = reset ? 0 : event.a;
        const int begin = std::max(previousFrame, event.frame / referenceBlock * referenceBlock);
        if (previousValue != value) {
            bends.push_back({begin, event.frame, previousValue, value});
            bends.push_back({event.frame, event.frame, value, value});
        }
        previousFrame = event.frame;
        previousValue = value;
    }
    return bends;
}

// Controller automation track (plan.cpp:136-216): block-aligned ramps to each
// new value, optionally smoothed in 16-frame groups.
template <class Transform>
Track automation(const Midi& midi, int cc, float initial, int smoothFrames, Transform transform, bool settle = false)
{
    float previous = transform(initial);
    Track points{{0, previous, 0}};
    struct Ramp { int first, last; float from, to; };
    std::vector<Ramp> ramps;
    int last = 0;
    for (const auto& event : midi.events) {
        float value = 0;
        if (event.kind == EventKind::control && event.a == 121) value = initial;
        else if (cc == 128 && event.kind == EventKind::bend) value = float(event.a);
        else if (event.kind == EventKind::control && event.a == cc) value = float(event.b);
        else continue;
        const float target = transform(value);
        if (settle && event.frame == 0) {
            points.front().value = target;
        } else if (target != previous) {
            const int first = std::max(last, event.frame / referenceBlock * referenceBlock);
            ramps.push_back({first, event.frame, previous, target});
        }
        previous = target;
        last = event.frame;
    }
    const auto add = [&](int frame, float value, float step) {
        if (points.back().frame == frame) {
            points.back() = {frame, value, step};
        } else if (points.back().step != step ||
                   std::abs(points.back().value + float(frame - points.back().frame) * step - value) > 1e-6f) {
            points.push_back({frame, value, step});
        }
    };
    if (smoothFrames < 2) {
        for (const auto& ramp : ramps) {
            if (ramp.first < ramp.last)
                add(ramp.first, ramp.from, (ramp.to - ramp.from) / float(ramp.last - ramp.first));
            add(ramp.last, ramp.to, 0);
        }
        return points;
    }
    float current = points.front().value, target = current, step = 0;
    size_t next = 0;
    constexpr int group = 16;
    const int smooth = std::max(group, smoothFrames);
    for (int frame = 0; next < ramps.size() || current != target; frame += group) {
        if (current == target && next < ramps.size() && frame < ramps[next].first)
            frame = std::max(frame, ramps[next].first / group * group);
        float nextTarget = target;
        const int end = frame + group - 1;
        while (next < ramps.size() && end >= ramps[next].last)
            nextTarget = ramps[next++].to;
        if (next < ramps.size() && end >= ramps[next].first) {
            const auto& ramp = ramps[next];
            nextTarget = ramp.from + (ramp.to - ramp.from) * (float(end - ramp.first) / float(ramp.last - ramp.first));
        }
        if (nextTarget != target) {
            target = nextTarget;
            step = (target - current) / float(smooth);
        }
        if (current == target || step == 0) {
            add(frame, current, 0);
            continue;
        }
        add(frame, current + step, step);
        const float limit = std::abs((target - current) / step);
        if (limit <= group) {
            add(frame + std::max(0, int(std::ceil(limit)) - 1), target, 0);
            current = target;
        } else {
            current += group * step;
        }
    }
    return points;
}

// The render path's envelope (render.cu:6-19 / plan.cpp:218-235), on the host.
template <class Envelope>
float envelopeValue(const Envelope& e, int frame)
{
    if (e.releaseStart >= 0 && frame >= e.releaseStart) {
        if (frame >= e.fadeStart)
            return std::max(0.f, e.fadeValue - float(frame - e.fadeStart + 1) * e.fadeStep);
        return e.releaseValue * std::exp(float(frame - e.releaseStart + 1) * e.releaseRate);
    }
    if (frame < e.attackStart) return e.start;
    if (frame < e.holdStart) return std::min(1.f, e.start + float(frame - e.attackStart + 1) * e.attackStep);
    if (frame < e.decayStart) return 1;
    if (e.decayRate == 0) return e.sustain;
    return std::max(e.sustain, std::exp(float(frame - e.decayStart + 1) * e.decayRate));
}

// Exponential release to -80 dB, then a 50 ms linear fade (plan.cpp:238-248).
template <class Envelope>
void releaseFrom(Envelope& e, int frame, int rate, float level, float seconds)
{
    e.releaseStart = frame;
    e.releaseValue = level;
    e.releaseRate = -9 / (std::clamp(seconds, .006f, 100.f) * float(rate));
    const int duration = level > silence ? static_cast<int>(std::log(silence / level) / e.releaseRate) : 0;
    e.fadeStart = frame + duration;
    e.fadeValue = level * std::exp(e.releaseRate * float(duration));
    e.fadeStep = std::max(silence, e.fadeValue) / (float(rate) * .05f);
}

double travel(const cs_voice_span& v, int frames)
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

// Last frame a voice can sound: the envelope's end, or the source end at the
// slowest pitch the voice can reach (plan.cpp:264-280).
int spanEnd(const cs_voice_span& v, int envelopeEnd)
{
    if (v.loopEnd > 0 || v.generator != CS_GEN_NONE)
        return envelopeEnd;
    const int rampFrames = std::max(0, v.bendEnd - v.begin);
    const double rampTravel = travel(v, rampFrames);
    const double remaining = v.sourceEnd - v.position;
    const double step = v.step * v.minimumPitchRatio;
    const double length = rampFrames && v.pitchSlope != 0 && remaining <= rampTravel
        ? std::ceil(std::log1p(std::max(0., remaining) * std::expm1(v.pitchSlope) / step) / v.pitchSlope)
        : rampFrames + std::ceil((remaining - rampTravel) / (step * std::exp(v.pitchSlope * rampFrames)));
    if (length > forever - v.begin)
        return envelopeEnd;
    return std::min(envelopeEnd, v.begin + std::max(0, static_cast<int>(length)));
}

class Planner {
public:
    Planner(const Instrument& instrument, SampleBank& bank, int rate, unsigned seed, int limit, TailPolicy tail)
        : instrument_(instrument), bank_(bank), rate_(rate), limit_(limit), tail_(tail), cc_(instrument.initialCC),
          sequence_(instrument.regions.size()), random_(seed), variation_(seed ^ 0x85ebca6b),
          currentSwitch_(instrument.initialSwitch)
    {
    }

    Plan run(const Midi& midi)
    {
        midi_ = &midi;
        hasBend_ = std::any_of(midi.events.begin(), midi.events.end(),
                               [](const Event& e) { return e.kind == EventKind::bend && e.a != 0; });
        for (int cc : {7, 11, 10}) {
            if (instrument_.usedCC[size_t(cc)]) {
                plan_.controls.push_back({{0, cc == 10 ? 0.f : 1.f, 0}});
            } else {
                const int curve = cc == 10 ? 1 : 4;
                plan_.controls.push_back(automation(midi, cc, instrument_.initialCC[size_t(cc)], rate_ / 100,
                    [&](float value) { return curveValue(instrument_, curve, value); }, tail_ == TailPolicy::natural));
            }
        }
        const auto bends = bendRamps(midi);
        size_t nextBend = 0;
        for (const auto& event : midi.events) {
            while (nextBend < bends.size() && bends[nextBend].begin <= event.frame)
                changeBend(bends[nextBend++]);
            prune(event.frame);
            switch (event.kind) {
            case EventKind::on: noteOn(event); break;
            case EventKind::off: noteOff(event); break;
            case EventKind::control: control(event); break;
            case EventKind::bend: break;
            }
        }
        prune(midi.end);
        for (auto& voice : active_) {
            // Natural mode ends notes through the prepared MIDI and its pedal releases.
            if (tail_ != TailPolicy::natural && voice.kind == VoiceKind::attack && voice.region->loop != LoopMode::oneShot)
                release(voice, midi.end);
            if (voice.span.end == forever && limit_ == forever)
                throw std::runtime_error("a looping one-shot or release sample has no finite end");
            emit(voice.span, voice.span.end);
        }
        if (tail_ != TailPolicy::natural)
            plan_.frames = std::max(plan_.frames, midi.end);
        if (plan_.spans.empty())
            throw std::runtime_error("no playable notes for this SFZ and MIDI");
        buildLfoTracks();
        return std::move(plan_);
    }

private:
    void emit(cs_voice_span span, int end)
    {
        span.end = std::min(span.end, end);
        plan_.tailClipped |= span.end > limit_ && span.begin < span.end;
        span.end = std::min(span.end, limit_);
        if (span.begin < span.end) {
            for (int i = span.firstLfo; i < span.firstLfo + span.lfoCount; ++i)
                lfos_[size_t(i)].end = std::max(lfos_[size_t(i)].end, span.end);
            plan_.frames = std::max(plan_.frames, span.end);
            plan_.spans.push_back(span);
        }
    }

    void prune(int frame)
    {
        const auto tail = std::remove_if(active_.begin(), active_.end(), [&](const Voice& voice) {
            if (voice.span.end > frame)
                return false;
            emit(voice.span, voice.span.end);
            return true;
        });
        active_.erase(tail, active_.end());
    }

    void split(Voice& voice, int frame, double position)
    {
        emit(voice.span, frame);
        voice.span.begin = frame;
        voice.span.position = position;
    }

    bool pedal(const Region& region) const
    {
        return region.sustainEnabled && cc_[size_t(region.sustainCC)] >= region.sustainLow;
    }

    bool matches(const Region& r, int velocity, float draw) const
    {
        return velocity >= r.lowVelocity && velocity <= r.highVelocity && draw >= r.randomLow &&
            draw < r.randomHigh && switchesMatch(r) && controllersMatch(r);
    }

    bool switchesMatch(const Region& r) const
    {
        return (r.switchLow < 0 || (currentSwitch_ >= r.switchLow && currentSwitch_ <= r.switchHigh)) &&
            (r.switchDown < 0 || down_[size_t(r.switchDown)]) && (r.switchUp < 0 || !down_[size_t(r.switchUp)]) &&
            (r.switchPrevious < 0 || previousNote_ == r.switchPrevious);
    }

    bool controllersMatch(const Region& r) const
    {
        return std::all_of(r.conditions.begin(), r.conditions.end(), [&](const Condition& c) {
            return cc_[c.cc] >= c.low && cc_[c.cc] <= c.high;
        });
    }

    void applyBend(Voice& voice) const
    {
        cs_voice_span& span = voice.span;
        if (voice.region->bendSmooth > 0) {
            span.bendEnd = span.begin;
            span.pitchSlope = 0;
            span.step = voice.baseStep;
            return;
        }
        const auto cents = [&](int value) {
            const double normalized = std::max(-8191, value) / 8191.0;
            return normalized >= 0 ? normalized * voice.region->bendUp : -normalized * voice.region->bendDown;
        };
        const double to = cents(bend_.to);
        span.bendEnd = bend_.end;
        span.pitchSlope = 0;
        if (span.begin < bend_.end) {
            const double from = cents(bend_.from);
            const double slope = (to - from) / (bend_.end - bend_.begin);
            span.pitchSlope = slope * (std::log(2.) / 1200);
            span.step = voice.baseStep * std::exp2((from + (span.begin - bend_.begin) * slope) / 1200);
        } else {
            span.step = voice.baseStep * std::exp2(to / 1200);
        }
    }

    void changeBend(const Bend& bend)
    {
        prune(bend.begin);
        bend_ = bend;
        for (auto& voice : active_) {
            if (voice.region->bendSmooth > 0)
                continue;
            const int start = std::max(bend.begin, voice.span.begin);
            const double phase = voice.span.position + travel(voice.span, start - voice.span.begin);
            split(voice, start, phase);
            applyBend(voice);
            voice.span.end = spanEnd(voice.span, fadeEnd(voice.span));
        }
    }

    int fadeEnd(const cs_voice_span& span) const
    {
        return span.releaseStart < 0 ? forever : span.fadeStart + rate_ / 20 + 1;
    }

    float controllerValue(const Modulation& mod, int key, int velocity, VoiceKind kind) const
    {
        if (mod.cc == 140) return keyDelta_;
        if (mod.cc == 141) return std::abs(keyDelta_);
        float value = 0;
        if (mod.cc < 128) value = cc_[size_t(mod.cc)];
        else if (mod.cc == 133) value = float(key);
        else if ((mod.cc == 131 && kind == VoiceKind::attack) || (mod.cc == 132 && kind == VoiceKind::release))
            value = float(velocity);
        else if (mod.cc == 134) value = keysDown_ > 0 ? 127.f : 0.f;
        else if (mod.cc == 135) value = 127 * randomValue_;
        else if (mod.cc == 136) value = 127 * (2 * randomValue_ - 1);
        else if (mod.cc == 137) value = alternate_ ? 127.f : 0.f;
        else if (const auto it = instrument_.extendedCCDefaults.find(mod.cc); it != instrument_.extendedCCDefaults.end())
            value = it->second;
        return curveValue(instrument_, mod.curve, value);
    }

    int controllerTrack(const Modulation& mod)
    {
        const auto key = std::make_tuple(mod.cc, mod.curve, mod.smooth);
        const auto result = tracks_.emplace(key, int(plan_.controls.size()));
        if (result.second)
            plan_.controls.push_back(automation(*midi_, mod.cc, instrument_.initialCC[size_t(mod.cc)],
                mod.smooth * rate_ / 1000, [&](float value) { return curveValue(instrument_, mod.curve, value); },
                tail_ == TailPolicy::natural));
        return result.first->second;
    }

    int smoothBendTrack(const Region& region)
    {
        const auto key = std::make_tuple(region.bendUp, region.bendDown, region.bendSmooth);
        const auto result = bendTracks_.emplace(key, int(plan_.controls.size()));
        if (result.second)
            plan_.controls.push_back(automation(*midi_, 128, 0, region.bendSmooth * rate_ / 1000,
                [&](float value) {
                    const float bend = std::max(-8191.f, value) / 8191;
                    return bend >= 0 ? bend * region.bendUp : -bend * region.bendDown;
                }, tail_ == TailPolicy::natural));
        return result.first->second;
    }

    int controllerFadeTrack(int cc, const Crossfade& fade)
    {
        const auto key = std::make_tuple(cc, fade.inLow, fade.inHigh, fade.outLow, fade.outHigh, fade.power);
        const auto result = fadeTracks_.emplace(key, int(plan_.controls.size()));
        if (result.second)
            plan_.controls.push_back(automation(*midi_, cc, instrument_.initialCC[size_t(cc)], rate_ / 200,
                [&](float value) { return crossfadeGain(fade, value, true); }, tail_ == TailPolicy::natural));
        return result.first->second;
    }

    float param(const Region& r, int target, float base, int key, int velocity, VoiceKind kind) const
    {
        if (target >= CS_MOD_ENV_DELAY && target <= CS_MOD_ENV_RELEASE)
            base += r.velocityEnvelope[size_t(target - CS_MOD_ENV_DELAY)] * (float(velocity) / 127.f);
        for (const auto& m : r.modulation)
            if (m.target == target)
                base += m.depth * controllerValue(m, key, velocity, kind);
        return base;
    }

    void initSecondary(Voice& voice)
    {
        cs_voice_span& span = voice.span;
        for (int slot = 0; slot < 2; ++slot) {
            const auto& source = voice.region->secondary[size_t(slot)];
            if (!source.enabled)
                continue;
            const int first = slot == 0 ? CS_MOD_FILEG_DELAY : CS_MOD_PITCHEG_DELAY;
            std::array<float, 7> values;
            for (size_t p = 0; p < values.size(); ++p) {
                const float base = source.values[p] + source.velocity[p] * (float(voice.velocity) / 127.f);
                const float value = param(*voice.region, first + int(p), base, voice.key, voice.velocity, voice.kind);
                values[p] = std::clamp(value, 0.f, p == 4 || p == 5 ? 1.f : 100.f);
            }
            cs_envelope_shape& shape = span.extraEnvelope[slot];
            span.activeEnvelope[slot] = 1;
            shape.start = values[5];
            shape.attackStart = span.begin + int(values[0] * float(rate_));
            const float attack = values[1] * float(rate_);
            shape.attackStep = attack > 0 ? 1 / attack : 1;
            shape.holdStart = shape.attackStart + std::max(0, int(std::ceil((1 - shape.start) * attack)) - 1);
            shape.decayStart = shape.holdStart + int(values[2] * float(rate_));
            shape.decayRate = values[3] > 0 ? -9 / (std::max(.006f, values[3]) * float(rate_)) : 0;
            shape.sustain = values[4];
            shape.releaseStart = -1;
            shape.releaseSeconds = values[6];
            shape.depth = source.depth + source.velocityDepth * (float(voice.velocity) / 127.f);
        }
    }

    float appendLfos(Voice& voice, int frame, bool& modulatedStereo)
    {
        cs_voice_span& span = voice.span;
        span.firstLfo = int(lfos_.size());
        float pitchBound = 0;
        for (const auto& [index, lfo] : voice.region->lfos) {
            (void)index;
            LfoTrack track{&lfo, frame, frame, 0, 0, {}, {}};
            float delay = lfo.delay, fade = lfo.fade;
            auto bounds = lfo.depths;
            for (auto& depth : bounds)
                depth.second = std::abs(depth.second);
            for (const auto& m : lfo.modulation) {
                const float value = controllerValue(m, voice.key, voice.velocity, voice.kind);
                if (m.target == CS_MOD_LFO_DELAY) {
                    delay += m.depth * value;
                } else if (m.target == CS_MOD_LFO_FADE) {
                    fade += m.depth * value;
                } else {
                    const int source = m.cc < 128 ? controllerTrack(m) : -1;
                    track.inputs.push_back({source, 0, m.target, source < 0 ? m.depth * value : m.depth, -1, 0});
                    if (m.target < CS_MOD_LFO_FREQUENCY || m.target >= CS_MOD_EQ1_FREQUENCY) {
                        float maximum = std::abs(value);
                        if (source >= 0)
                            for (const auto& point : plan_.controls[size_t(source)])
                                maximum = std::max(maximum, std::abs(point.value));
                        bounds[m.target] += std::abs(m.depth) * maximum;
                    }
                }
            }
            track.delay = int(std::clamp(delay, 0.f, 100.f) * float(rate_));
            track.fade = int(std::clamp(fade, 0.f, 100.f) * float(rate_));
            for (const auto& [target, bound] : bounds) {
                if (bound == 0)
                    continue;
                modulatedStereo |= target == CS_MOD_WIDTH || target == CS_MOD_POSITION;
                if (target == CS_MOD_PITCH)
                    pitchBound += bound;
                const int trackIndex = int(plan_.controls.size());
                plan_.controls.emplace_back();
                track.outputs.emplace_back(target, trackIndex);
                plan_.modulation.push_back({trackIndex, 0, target, 1, -1, 0});
            }
            if (!track.outputs.empty())
                lfos_.push_back(std::move(track));
        }
        span.lfoCount = int(lfos_.size()) - span.firstLfo;
        return pitchBound;
    }

    // LFO outputs sampled every 16 frames (sine/triangle) or every frame, as
    // piecewise-linear tracks (plan.cpp:589-639).
    void buildLfoTracks()
    {
        std::mt19937 sampleHold(1);
        for (const auto& lfo : lfos_) {
            const Lfo& source = *lfo.source;
            const int start = lfo.begin + lfo.delay;
            const int stride = source.wave <= 1 ? 16 : 1;
            double phase = 0;
            int cycle = -1;
            float held = 0;
            std::array<float, CS_MOD_EQ3_GAIN + 1> baseDepth{};
            for (const auto& [target, depth] : source.depths)
                baseDepth[size_t(target)] = depth;
            for (const auto& output : lfo.outputs)
                plan_.controls[size_t(output.second)].push_back({0, 0, 0});
            for (int frame = start; frame < lfo.end; frame += stride) {
                float frequency = source.frequency, shift = source.phase;
                auto depth = baseDepth;
                for (const auto& m : lfo.inputs) {
                    const float value = m.first < 0 ? m.depth : m.depth * valueAt(plan_.controls[size_t(m.first)], frame);
                    if (m.target == CS_MOD_LFO_FREQUENCY) frequency += value;
                    else if (m.target == CS_MOD_LFO_PHASE) shift += value;
                    else depth[size_t(m.target)] += value;
                }
                float wave = lfoShape(source.wave, phase + shift);
                if (source.wave == 12) {
                    const int nextCycle = static_cast<int>(phase);
                    if (cycle != nextCycle) {
                        held = 2 * std::generate_canonical<float, 24>(sampleHold) - 1;
                        cycle = nextCycle;
                    }
                    wave = held;
                }
                const float fade = lfo.fade == 0 ? 1.f : std::min(1.f, float(frame - start) / float(lfo.fade));
                for (const auto& output : lfo.outputs) {
                    Track& points = plan_.controls[size_t(output.second)];
                    const float value = depth[size_t(output.first)] * wave * fade;
                    if (points.back().frame == frame) {
                        points.back().value = value;
                    } else {
                        if (stride > 1 && frame - points.back().frame == stride)
                            points.back().step = (value - points.back().value) / float(stride);
                        if (stride > 1 || value != points.back().value)
                            points.push_back({frame, value, 0});
                    }
                }
                phase += double(std::clamp(frequency, 0.f, 1000.f)) * stride / rate_;
            }
        }
    }

    float appendPitchEnvelopes(Voice& voice)
    {
        float bound = 0;
        for (const auto& [id, source] : voice.region->pitchEnvelopes) {
            (void)id;
            std::vector<cs_voice_modulation> bindings;
            if (source.depth != 0) {
                bindings.push_back({-1, 0, CS_MOD_PITCH, source.depth, -1, 0});
                bound += std::abs(source.depth);
            }
            for (const auto& [cc, depth] : source.depthCC) {
                const Modulation m{CS_MOD_PITCH, cc, depth};
                const float value = controllerValue(m, voice.key, voice.velocity, voice.kind);
                if (cc < 128) {
                    bindings.push_back({controllerTrack(m), 0, CS_MOD_PITCH, depth, -1, 0});
                    bound += std::abs(depth);
                } else if (value != 0) {
                    bindings.push_back({-1, 0, CS_MOD_PITCH, depth * value, -1, 0});
                    bound += std::abs(depth * value);
                }
            }
            if (bindings.empty())
                continue;
            const int shape = int(plan_.controls.size());
            voice.flexShapes.push_back(shape);
            Track& track = plan_.controls.emplace_back();
            track.push_back({0, 0, 0});
            const auto write = [&](int frame, float level, float step) {
                if (track.back().frame == frame) track.back() = {frame, level, step};
                else track.push_back({frame, level, step});
            };
            int frame = voice.triggerFrame;
            float level = 0;
            for (const auto& [index, point] : source.points) {
                (void)index;
                float time = point.seconds;
                for (const auto& [cc, seconds] : point.timeCC)
                    time += seconds * controllerValue({CS_MOD_PITCH, cc}, voice.key, voice.velocity, voice.kind);
                const int frames = int(std::clamp(time, 0.f, 100.f) * float(rate_));
                if (frames > 0)
                    write(frame, level, (point.level - level) / float(frames));
                level = point.level;
                frame += frames;
                write(frame, level, 0);
            }
            for (auto b : bindings) {
                b.shapeFirst = shape;
                plan_.modulation.push_back(b);
            }
        }
        return bound;
    }

    void trigger(const Region& r, int frame, int key, int velocity, VoiceKind kind, int duration = 0,
                 int controller = -1)
    {
        if (instrument_.hasOffBy)
            choke(r, frame, controller >= 0 ? controller : key, kind);
        if (r.notePolyphony)
            limitNoteVoices(r, frame, key, velocity);
        const Sample* sample = r.generator == CS_GEN_NONE ? &bank_.decode(r.sample) : nullptr;
        const auto vary = [&](float extent) {
            return extent == 0 ? 0.f : extent * std::generate_canonical<float, 24>(variation_);
        };
        Voice voice{};
        voice.key = key;
        voice.velocity = velocity;
        voice.triggerFrame = frame;
        voice.region = &r;
        voice.kind = kind;
        const auto modulated = [&](int target, float base) { return param(r, target, base, key, velocity, kind); };
        const auto seconds = [&](int target, float base) { return std::clamp(modulated(target, base), 0.f, 100.f); };
        voice.releaseSeconds = seconds(CS_MOD_ENV_RELEASE, r.release);
        const double baseRate = sample ? sample->rate : 440 * std::exp2((r.rootKey - 69) / 12.);
        voice.baseStep = (baseRate / rate_) * std::exp2(
            (r.keyTrack * (key - r.rootKey) + r.tune + 100 * r.transpose + vary(r.pitchRandom)) / 1200.0);
        cs_voice_span& span = voice.span;
        span.sample = sample ? sample->offset : 0;
        span.channels = sample ? sample->channels : 1;
        span.generator = r.generator;
        if (r.generator == CS_GEN_NOISE) {
            span.noiseSeed = variation_();
            span.noiseStart = frame;
        }
        span.begin = frame + int(seconds(CS_MOD_DELAY, r.delay) * float(rate_));
        span.sourceEnd = r.end;
        const int randomizedOffset = r.offsetRandom ? std::uniform_int_distribution<int>(0, r.offsetRandom)(variation_) : 0;
        if (sample) {
            span.position = std::trunc(std::clamp(double(modulated(CS_MOD_OFFSET, float(r.offset))) + randomizedOffset,
                                                  0., double(r.end)));
        } else {
            const float phase = r.oscillatorPhase >= 0 ? r.oscillatorPhase : randomValue_;
            span.position = phase - std::floor(phase);
        }
        applyBend(voice);
        if (sample && (r.loop == LoopMode::continuous || r.loop == LoopMode::sustain)) {
            span.loopFirst = r.loopStart;
            span.loopEnd = r.loopEnd;
            span.loopCrossfade = static_cast<int>(std::lround(std::min<double>(r.loopStart,
                                                                                double(r.loopCrossfade) * sample->rate)));
        }
        span.start = std::clamp(modulated(CS_MOD_ENV_START, r.start), 0.f, 1.f);
        span.attackStart = span.begin + int(seconds(CS_MOD_ENV_DELAY, r.envelopeDelay) * float(rate_));
        const float attackFrames = seconds(CS_MOD_ENV_ATTACK, r.attack) * float(rate_);
        span.attackStep = attackFrames > 0 ? 1 / attackFrames : 1;
        span.holdStart = span.attackStart + std::max(0, int(std::ceil((1 - span.start) * attackFrames)) - 1);
        span.decayStart = span.holdStart + int(seconds(CS_MOD_ENV_HOLD, r.hold) * float(rate_));
        const float decay = seconds(CS_MOD_ENV_DECAY, r.decay);
        span.decayRate = decay > 0 ? -9 / (std::max(.006f, decay) * float(rate_)) : 0;
        span.sustain = std::clamp(modulated(CS_MOD_ENV_SUSTAIN, r.sustain), 0.f, 1.f);
        span.releaseStart = -1;
        initSecondary(voice);
        span.filterTrack = -1;
        span.sampleRate = rate_;
        for (size_t i = 0; i < r.filters.size(); ++i) {
            const Filter& filter = r.filters[i];
            if (filter.type == CS_FILTER_NONE)
                continue;
            if (span.filterTrack < 0)
                span.filterTrack = plan_.filterTracks++;
            const int velocityTarget = i == 0 ? CS_MOD_FILTER_VELOCITY : CS_MOD_FILTER_VELOCITY2;
            const float cents = filter.keyTrack * float(key - filter.keyCenter) + vary(filter.random) +
                modulated(velocityTarget, filter.velocityTrack) * float(velocity) / 127.f;
            span.filters[i] = {filter.type,
                std::clamp(filter.cutoff * std::exp2(std::clamp(cents, -24000.f, 24000.f) / 1200), 0.f, 20000.f),
                filter.resonance, 0, 0};
        }
        constexpr float eqDefaults[] = {50, 500, 5000};
        for (size_t i = 0; i < r.eq.size(); ++i) {
            const Equalizer& eq = r.eq[i];
            if (!eq.enabled)
                continue;
            if (span.filterTrack < 0)
                span.filterTrack = plan_.filterTracks++;
            span.filters[i + 2] = {CS_FILTER_PEAK, eq.frequency == 0 ? eqDefaults[i] : eq.frequency, 0, eq.bandwidth,
                                   eq.gain};
        }
        span.firstModulation = int(plan_.modulation.size());
        bool modulatedStereo = false;
        float pitchBound = std::abs(span.extraEnvelope[1].depth);
        for (const auto& m : r.modulation) {
            if ((m.target >= CS_MOD_ENV_DELAY && m.target < CS_MOD_CUTOFF) ||
                (m.target >= CS_MOD_FILTER_VELOCITY && m.target < CS_MOD_FILEG_DEPTH))
                continue;
            modulatedStereo |= m.target == CS_MOD_WIDTH || m.target == CS_MOD_POSITION;
            if (m.target == CS_MOD_PITCH || m.target == CS_MOD_PITCHEG_DEPTH)
                pitchBound += std::abs(m.cc < 128 ? m.depth : m.depth * controllerValue(m, key, velocity, kind));
            if (m.cc < 128)
                plan_.modulation.push_back({controllerTrack(m), 0, m.target, m.depth, -1, 0});
            else
                plan_.modulation.push_back({-1, 0, m.target, m.depth * controllerValue(m, key, velocity, kind), -1, 0});
        }
        for (const auto& [cc, fade] : r.controllerFades)
            plan_.modulation.push_back({controllerFadeTrack(cc, fade), 0, CS_MOD_AMPLITUDE, 1, -1, 0});
        if (r.bendSmooth > 0 && hasBend_) {
            pitchBound += std::max(std::abs(r.bendUp), std::abs(r.bendDown));
            plan_.modulation.push_back({smoothBendTrack(r), 0, CS_MOD_PITCH, 1, -1, 0});
        }
        pitchBound += appendLfos(voice, frame, modulatedStereo);
        pitchBound += appendPitchEnvelopes(voice);
        span.minimumPitchRatio = std::exp2(-std::min(24000.f, pitchBound) / 1200);
        if (pitchBound > 0) {
            span.variablePitch = 1;
            if (span.filterTrack < 0)
                span.filterTrack = plan_.filterTracks++;
        }
        span.modulationCount = int(plan_.modulation.size()) - span.firstModulation;
        const float noteGain = kind == VoiceKind::controller ? 1.f : velocityGain(r, velocity) *
            crossfadeGain(r.keyFade, float(key), false) * crossfadeGain(r.velocityFade, float(velocity), true);
        const float gain = r.amplitude * noteGain *
            std::pow(10.f, ((tail_ == TailPolicy::natural ? 0 : masterGainDb) + r.volume + vary(r.ampRandom) -
                            r.releaseDecay * float(duration) / float(rate_) + 3) / 20);
        const bool stereoMatrix = span.channels == 2 && (modulatedStereo || r.width != 1 || r.position != 0);
        span.stereoMatrix = stereoMatrix;
        const float positionGain = span.channels == 1 ? 1.f : .99881488f;
        span.gain = gain * (stereoMatrix ? panCompensation : positionGain);
        span.pan = r.pan;
        span.width = r.width;
        span.stereoPosition = r.position;
        span.left = span.gain * std::cos((1 + r.pan) * quarterPi);
        span.right = span.gain * std::cos((1 - r.pan) * quarterPi);
        span.widthDirect = stereoMatrix ? std::cos((1 - r.width) * quarterPi) : 1.f;
        span.widthCross = stereoMatrix ? std::cos((1 + r.width) * quarterPi) : 0.f;
        span.positionLeft = stereoMatrix ? std::cos((1 + r.position) * quarterPi) : 1.f;
        span.positionRight = stereoMatrix ? std::cos((1 - r.position) * quarterPi) : 1.f;
        span.end = spanEnd(span, forever);
        active_.push_back(voice);
    }

    void release(Voice& voice, int frame)
    {
        if (voice.span.releaseStart >= 0 || voice.kind != VoiceKind::attack || voice.region->loop == LoopMode::oneShot)
            return;
        if (voice.region->envelopeDynamic)
            voice.releaseSeconds = param(*voice.region, CS_MOD_ENV_RELEASE, voice.region->release, voice.key,
                                         voice.velocity, voice.kind);
        startRelease(voice, frame, voice.releaseSeconds);
    }

    void startRelease(Voice& voice, int frame, float seconds)
    {
        cs_voice_span& span = voice.span;
        if (frame >= span.end)
            return;
        if (frame < span.begin) {
            span.end = span.begin;
            return;
        }
        const float level = envelopeValue(span, frame - 1);
        const bool exitLoop = voice.region->loop == LoopMode::sustain && span.loopEnd > 0;
        if (exitLoop || span.releaseStart >= 0) {
            const double phase = span.position + travel(span, frame - span.begin);
            split(voice, frame, exitLoop ? wrapped(span, phase) : phase);
            applyBend(voice);
            if (exitLoop)
                span.loopEnd = 0;
        }
        releaseFrom(span, frame, rate_, level, seconds);
        for (int shape : voice.flexShapes) {
            Track& track = plan_.controls[size_t(shape)];
            track.erase(std::lower_bound(track.begin(), track.end(), frame,
                [](const cs_control_point& point, int value) { return point.frame < value; }), track.end());
            track.push_back({frame, 0, 0});
        }
        for (int slot = 0; slot < 2; ++slot) {
            cs_envelope_shape& shape = span.extraEnvelope[slot];
            if (span.activeEnvelope[slot] && shape.releaseStart < 0)
                releaseFrom(shape, frame, rate_, envelopeValue(shape, frame - 1), shape.releaseSeconds);
        }
        span.end = spanEnd(span, fadeEnd(span));
    }

    void choke(const Region& incoming, int frame, int key, VoiceKind cause)
    {
        std::vector<std::pair<int, int>> released;
        for (auto& voice : active_) {
            const Region& r = *voice.region;
            if (voice.span.end <= frame || voice.kind == VoiceKind::release || voice.choked || !r.chokedByGroup ||
                r.offBy != incoming.group || (r.group == incoming.group && voice.key == key && controllersMatch(r)))
                continue;
            forceOff(voice, frame);
            if (cause != VoiceKind::controller && voice.kind == VoiceKind::attack)
                released.emplace_back(voice.key, voice.velocity);
        }
        for (const auto& note : released)
            releaseRegions(frame, note.first, note.second, std::max(0, frame - noteStart_[size_t(note.first)]));
    }

    void forceOff(Voice& voice, int frame)
    {
        const Region& r = *voice.region;
        voice.choked = true;
        const float time = r.offMode == OffMode::normal ? voice.releaseSeconds : r.offMode == OffMode::fast ? .006f : r.offTime;
        startRelease(voice, frame, time);
    }

    void limitNoteVoices(const Region& region, int frame, int key, int velocity)
    {
        std::vector<Voice*> candidates;
        int count = 0;
        for (auto& voice : active_) {
            if (voice.choked || voice.span.end <= frame || voice.key != key || voice.region->group != region.group)
                continue;
            ++count;
            if (!region.selfMask || voice.velocity <= velocity)
                candidates.push_back(&voice);
        }
        if (count < region.notePolyphony)
            return;
        std::stable_sort(candidates.begin(), candidates.end(), [&](const Voice* a, const Voice* b) {
            return region.selfMask ? a->velocity < b->velocity : a->triggerFrame < b->triggerFrame;
        });
        for (Voice* candidate : candidates) {
            if (candidate->choked)
                continue;
            for (auto& sister : active_)
                if (!sister.choked && sister.key == candidate->key && sister.kind == candidate->kind &&
                    sister.triggerFrame == candidate->triggerFrame)
                    forceOff(sister, frame);
            if (--count < region.notePolyphony)
                break;
        }
    }

    void noteOn(const Event& event)
    {
        const bool switching = instrument_.switchKeys[size_t(event.a)];
        if (switching)
            currentSwitch_ = event.a;
        if (!down_[size_t(event.a)] && !switching)
            ++keysDown_;
        if (!switching) {
            keyDelta_ = lastNote_ < 0 ? 0.f : float(event.a - lastNote_);
            lastNote_ = event.a;
            randomValue_ = std::generate_canonical<float, 24>(extendedRandom_);
            alternate_ = !alternate_;
        }
        down_[size_t(event.a)] = true;
        noteVelocity_[size_t(event.a)] = event.b;
        noteStart_[size_t(event.a)] = event.frame;
        const float draw = std::generate_canonical<float, 24>(random_);
        for (const int index : instrument_.byKey[size_t(event.a)]) {
            const Region& region = instrument_.regions[size_t(index)];
            const bool step = sequence_[size_t(index)]++ % unsigned(region.sequenceLength) ==
                unsigned(region.sequencePosition - 1);
            if (!step || !matches(region, event.b, draw))
                continue;
            if (region.trigger == Trigger::attack || (region.trigger == Trigger::first && keysDown_ == 1) ||
                (region.trigger == Trigger::legato && keysDown_ > 1))
                trigger(region, event.frame, event.a, event.b, VoiceKind::attack);
        }
        previousNote_ = event.a;
    }

    bool hasAttackVoice(const Region& r) const
    {
        return std::any_of(active_.begin(), active_.end(), [&](const Voice& voice) {
            return voice.kind == VoiceKind::attack && voice.key >= r.lowKey && voice.key <= r.highKey &&
                voice.velocity >= r.lowVelocity && voice.velocity <= r.highVelocity;
        });
    }

    void noteOff(const Event& event)
    {
        if (!down_[size_t(event.a)])
            return;
        down_[size_t(event.a)] = false;
        if (!instrument_.switchKeys[size_t(event.a)])
            --keysDown_;
        for (auto& voice : active_) {
            if (voice.key == event.a && voice.kind == VoiceKind::attack) {
                voice.noteOff = true;
                if (!pedal(*voice.region) && !voice.sostenuto)
                    release(voice, event.frame);
            }
        }
        releaseRegions(event.frame, event.a, noteVelocity_[size_t(event.a)], event.frame - noteStart_[size_t(event.a)]);
    }

    void releaseRegions(int frame, int key, int velocity, int duration)
    {
        const float draw = std::generate_canonical<float, 24>(random_);
        for (const int index : instrument_.byKey[size_t(key)]) {
            const Region& r = instrument_.regions[size_t(index)];
            const unsigned counter = sequence_[size_t(index)];
            const bool sequenceMatches = counter == 0 ? !r.explicitSequencePosition
                : (counter - 1) % unsigned(r.sequenceLength) == unsigned(r.sequencePosition - 1);
            if ((r.trigger != Trigger::release && r.trigger != Trigger::releaseKey) || !sequenceMatches ||
                !matches(r, velocity, draw))
                continue;
            if (r.trigger == Trigger::release && (pedal(r) || sostenutoKeys_[size_t(key)]))
                delayed_.push_back({key, velocity, duration, &r, sostenutoKeys_[size_t(key)]});
            else if (r.trigger == Trigger::releaseKey || r.releaseDead || hasAttackVoice(r))
                trigger(r, frame, key, velocity, VoiceKind::release, duration);
        }
    }

    void updateDynamicEnvelopes(const std::array<float, 128>& before, int frame)
    {
        for (auto& voice : active_) {
            if (voice.choked)
                continue;
            for (const auto& mod : voice.region->modulation) {
                if (mod.cc >= 128 || before[size_t(mod.cc)] == cc_[size_t(mod.cc)] || mod.depth == 0)
                    continue;
                const bool filter = mod.target >= CS_MOD_FILEG_DELAY && mod.target <= CS_MOD_FILEG_RELEASE;
                const bool pitch = mod.target >= CS_MOD_PITCHEG_DELAY && mod.target <= CS_MOD_PITCHEG_RELEASE;
                if ((filter && voice.region->secondary[0].dynamic) || (pitch && voice.region->secondary[1].dynamic))
                    throw std::runtime_error("changing a dynamic pitch or filter envelope mid-voice is unsupported");
                if (!voice.region->envelopeDynamic || mod.target < CS_MOD_ENV_DELAY || mod.target > CS_MOD_ENV_RELEASE)
                    continue;
                if (mod.target != CS_MOD_ENV_RELEASE)
                    throw std::runtime_error("changing a dynamic amplitude envelope mid-voice is unsupported for CC" +
                                             std::to_string(mod.cc));
                if (voice.span.releaseStart >= 0 && frame < voice.span.fadeStart) {
                    const float seconds = param(*voice.region, CS_MOD_ENV_RELEASE, voice.region->release, voice.key,
                                                voice.velocity, voice.kind);
                    startRelease(voice, frame, seconds);
                    break;
                }
            }
        }
    }

    void control(const Event& event)
    {
        if (event.a == 121) {
            const auto before = cc_;
            cc_ = instrument_.initialCC;
            updateDynamicEnvelopes(before, event.frame);
            if (tail_ == TailPolicy::natural) {
                setSostenuto(false);
                releasePedals(event.frame, 66, before[66]);
            }
            for (auto& voice : active_)
                if (voice.noteOff && !pedal(*voice.region))
                    release(voice, event.frame);
            return;
        }
        const bool natural = tail_ == TailPolicy::natural;
        if (!natural && event.a == 66 && event.b != 0)
            throw std::runtime_error("unsupported MIDI sostenuto CC66");
        if (natural && (event.a == 120 || event.a == 123)) {
            for (auto& voice : active_)
                emit(voice.span, event.frame);
            active_.clear();
            delayed_.clear();
            down_.fill(false);
            sostenutoKeys_.fill(false);
            keysDown_ = 0;
            return;
        }
        if (event.a >= 120)
            throw std::runtime_error("unsupported MIDI channel mode CC" + std::to_string(event.a));
        const bool sostenuto = natural && event.a == 66;
        if (!instrument_.usedCC[size_t(event.a)] && !sostenuto)
            return;
        const auto before = cc_;
        const float previous = before[size_t(event.a)];
        cc_[size_t(event.a)] = float(event.b);
        if (previous != cc_[size_t(event.a)])
            updateDynamicEnvelopes(before, event.frame);
        if (sostenuto)
            setSostenuto(event.b == 127);
        releasePedals(event.frame, event.a, previous);
        const auto& triggers = instrument_.byCC[size_t(event.a)];
        if (triggers.empty())
            return;
        const float draw = std::generate_canonical<float, 24>(random_);
        for (const int index : triggers) {
            const Region& region = instrument_.regions[size_t(index)];
            const auto condition = std::find_if(region.ccTriggers.begin(), region.ccTriggers.end(),
                                                [&](const Condition& range) { return range.cc == event.a; });
            if (event.b < condition->low || event.b > condition->high || draw < region.randomLow ||
                draw >= region.randomHigh)
                continue;
            const bool step = sequence_[size_t(index)]++ % unsigned(region.sequenceLength) ==
                unsigned(region.sequencePosition - 1);
            if (step && switchesMatch(region) && previous != float(event.b) && controllersMatch(region))
                trigger(region, event.frame, region.rootKey, event.b, VoiceKind::controller, 0, event.a);
        }
    }

    void setSostenuto(bool down)
    {
        if (sostenutoDown_ == down)
            return;
        sostenutoDown_ = down;
        sostenutoKeys_ = down ? down_ : std::array<bool, 128>{};
        for (auto& voice : active_)
            voice.sostenuto = down && !voice.noteOff;
        if (!down)
            for (auto& note : delayed_)
                note.sostenuto = false;
    }

    void releasePedals(int frame, int cc, float previous)
    {
        const bool sostenutoUp = tail_ == TailPolicy::natural && cc == 66 && !sostenutoDown_;
        for (auto& voice : active_) {
            const Region& r = *voice.region;
            const bool sustainChanged = r.sustainEnabled && r.sustainCC == cc && previous >= r.sustainLow;
            if (voice.noteOff && (sustainChanged || sostenutoUp) && !pedal(r) && !voice.sostenuto)
                release(voice, frame);
        }
        std::vector<DelayedRelease> due;
        const auto end = std::remove_if(delayed_.begin(), delayed_.end(), [&](const DelayedRelease& note) {
            const Region& r = *note.region;
            if ((r.sustainCC != cc && !sostenutoUp) || pedal(r) || note.sostenuto)
                return false;
            if (r.releaseDead || hasAttackVoice(r))
                due.push_back(note);
            return true;
        });
        delayed_.erase(end, delayed_.end());
        for (const auto& note : due)
            trigger(*note.region, frame, note.key, note.velocity, VoiceKind::release, note.duration);
    }

    const Instrument& instrument_;
    SampleBank& bank_;
    int rate_, limit_;
    TailPolicy tail_;
    std::array<float, 128> cc_;
    std::array<bool, 128> down_{}, sostenutoKeys_{};
    bool sostenutoDown_ = false;
    std::array<int, 128> noteStart_{}, noteVelocity_{};
    std::vector<unsigned> sequence_;
    std::mt19937 random_, variation_;
    std::mt19937 extendedRandom_{1};
    std::vector<Voice> active_;
    std::vector<DelayedRelease> delayed_;
    int keysDown_ = 0, currentSwitch_;
    Bend bend_;
    const Midi* midi_ = nullptr;
    bool hasBend_ = false, alternate_ = false;
    int lastNote_ = -1, previousNote_ = -1;
    float keyDelta_ = 0, randomValue_ = 0;
    std::vector<LfoTrack> lfos_;
    std::map<std::tuple<int, int, int>, int> tracks_;
    std::map<std::tuple<float, float, int>, int> bendTracks_;
    std::map<std::tuple<int, int, int, int, int, bool>, int> fadeTracks_;
    Plan plan_;
};

} // namespace

Plan planRender(const Instrument& instrument, SampleBank& bank, const Midi& midi, int rate, unsigned seed, int limit,
                TailPolicy tail)
{
    return Planner(instrument, bank, rate, seed, limit, tail).run(midi);
}

} // namespace csh
