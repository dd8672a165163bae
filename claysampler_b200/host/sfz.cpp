// SFZ instrument loader.  Follows the reference's src/sfz/instrument.cpp: the
// same header scopes (<global>/<master>/<group>/<region>/<control>/<curve>),
// #define/#include, value ranges and opcode families, and the same rejection of
// unsupported opcodes, so that every instrument the reference accepts yields the
// same regions here (and every one it rejects is rejected with the same reason).
#include "host_types.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <stdexcept>
#include <string_view>

namespace csh {
namespace {

using Path = std::filesystem::path;
using Opcodes = std::map<std::string, std::string>;
constexpr std::string_view spaces = " \t\r\n";

std::string trimmed(std::string_view text)
{
    const auto first = text.find_first_not_of(spaces);
    if (first == text.npos)
        return {};
    const auto last = text.find_last_not_of(spaces);
    return std::string(text.substr(first, last - first + 1));
}

bool nameChar(char c) { return std::isalnum(static_cast<unsigned char>(c)) || c == '_'; }

std::string unquoted(std::string value)
{
    if (value.size() >= 2 && value.front() == '"' && value.back() == '"')
        return value.substr(1, value.size() - 2);
    return value;
}

Path pathOf(std::string value)
{
    std::replace(value.begin(), value.end(), '\\', '/');
    return std::filesystem::u8path(value);
}

float number(const std::string& value, float low, float high)
{
    size_t used = 0;
    const float result = std::stof(value, &used);
    if (used != value.size() || !std::isfinite(result) || result < low || result > high)
        throw std::runtime_error("invalid value " + value);
    return result;
}

int64_t integer64(const std::string& value, int64_t low, int64_t high)
{
    size_t used = 0;
    const auto result = std::stoll(value, &used);
    if (used != value.size() || result < low || result > high)
        throw std::runtime_error("invalid value " + value);
    return result;
}

int integer(const std::string& value, int low, int high) { return int(integer64(value, low, high)); }

// MIDI note number or a note name such as c#4 / Eb-1 (middle C = c4 = 60).
int noteNumber(const std::string& value)
{
    const int letter = value.empty() ? 0 : std::toupper(static_cast<unsigned char>(value[0]));
    if (value.size() < 2 || letter < 'A' || letter > 'G')
        return integer(value, 0, 127);
    constexpr int pitch[] = {9, 11, 0, 2, 4, 5, 7};
    int note = pitch[letter - 'A'];
    size_t octave = 1;
    if (value[octave] == '#' || value[octave] == 'b')
        note += value[octave++] == '#' ? 1 : -1;
    note += 12 * (integer(value.substr(octave), -2, 10) + 1);
    if (note < 0 || note > 127)
        throw std::runtime_error("key outside MIDI range " + value);
    return note;
}

bool onOff(const std::string& value)
{
    if (value == "on" || value == "1") return true;
    if (value == "off" || value == "0") return false;
    throw std::runtime_error("invalid switch " + value);
}

bool powerCurve(const std::string& value)
{
    if (value == "power") return true;
    if (value == "gain") return false;
    throw std::runtime_error("unsupported crossfade curve " + value);
}

bool isEnvelopeTarget(int target) { return target >= CS_MOD_ENV_DELAY && target <= CS_MOD_ENV_RELEASE; }

int controllerNumber(std::string_view suffix)
{
    const int cc = integer(std::string(suffix), 0, 511);
    if (cc >= 128 && cc <= 130)
        throw std::runtime_error("unsupported extended controller CC" + std::to_string(cc));
    return cc;
}

Modulation& binding(std::vector<Modulation>& list, int target, int cc)
{
    auto it = std::find_if(list.begin(), list.end(), [&](const Modulation& m) { return m.target == target && m.cc == cc; });
    if (it == list.end()) {
        list.push_back({target, cc});
        return list.back();
    }
    return *it;
}

// Splits "<field>ccN" style suffixes: 0 depth, 1 curve, 2 smooth, -1 none.
int ccField(std::string_view& suffix)
{
    const auto strip = [&](std::string_view prefix) {
        if (suffix.substr(0, prefix.size()) != prefix)
            return false;
        suffix.remove_prefix(prefix.size());
        return true;
    };
    if (strip("_oncc") || strip("_cc") || strip("cc")) return 0;
    if (strip("_curvecc")) return 1;
    if (strip("_smoothcc")) return 2;
    return -1;
}

// Controller-modulated region parameters (src/sfz/instrument.cpp:117-201).
bool modulationOpcode(Region& region, const std::string& op, const std::string& value, int envelopeShift = 0,
                      std::array<float, 7>* velocityEnvelope = nullptr)
{
    static const std::pair<std::string_view, int> parameters[] = {
        {"amplitude", CS_MOD_AMPLITUDE}, {"volume", CS_MOD_VOLUME}, {"gain", CS_MOD_VOLUME},
        {"pan", CS_MOD_PAN}, {"width", CS_MOD_WIDTH}, {"position", CS_MOD_POSITION},
        {"pitch", CS_MOD_PITCH}, {"tune", CS_MOD_PITCH},
        {"ampeg_delay", CS_MOD_ENV_DELAY}, {"ampeg_attack", CS_MOD_ENV_ATTACK},
        {"ampeg_hold", CS_MOD_ENV_HOLD}, {"ampeg_decay", CS_MOD_ENV_DECAY},
        {"ampeg_sustain", CS_MOD_ENV_SUSTAIN}, {"ampeg_start", CS_MOD_ENV_START},
        {"ampeg_release", CS_MOD_ENV_RELEASE}, {"offset", CS_MOD_OFFSET}, {"delay", CS_MOD_DELAY},
        {"cutoff", CS_MOD_CUTOFF}, {"cutoff1", CS_MOD_CUTOFF}, {"cutoff2", CS_MOD_CUTOFF2},
        {"resonance", CS_MOD_RESONANCE}, {"resonance1", CS_MOD_RESONANCE}, {"resonance2", CS_MOD_RESONANCE2},
        {"fil_veltrack", CS_MOD_FILTER_VELOCITY}, {"fil1_veltrack", CS_MOD_FILTER_VELOCITY},
        {"fil2_veltrack", CS_MOD_FILTER_VELOCITY2},
        {"eq1_freq", CS_MOD_EQ1_FREQUENCY}, {"eq1_bw", CS_MOD_EQ1_BANDWIDTH}, {"eq1_gain", CS_MOD_EQ1_GAIN},
        {"eq2_freq", CS_MOD_EQ2_FREQUENCY}, {"eq2_bw", CS_MOD_EQ2_BANDWIDTH}, {"eq2_gain", CS_MOD_EQ2_GAIN},
        {"eq3_freq", CS_MOD_EQ3_FREQUENCY}, {"eq3_bw", CS_MOD_EQ3_BANDWIDTH}, {"eq3_gain", CS_MOD_EQ3_GAIN},
    };
    const std::string_view opcode(op);
    for (const auto& [name, baseTarget] : parameters) {
        if (envelopeShift && !isEnvelopeTarget(baseTarget))
            continue;
        const int target = baseTarget + envelopeShift;
        if (isEnvelopeTarget(baseTarget) && baseTarget != CS_MOD_ENV_START &&
            (opcode == "ampeg_velto" + std::string(name.substr(6)) ||
             opcode == "ampeg_vel2" + std::string(name.substr(6)))) {
            const float depth = number(value, -100, 100);
            auto& velocity = velocityEnvelope ? *velocityEnvelope : region.velocityEnvelope;
            velocity[size_t(baseTarget - CS_MOD_ENV_DELAY)] = baseTarget == CS_MOD_ENV_SUSTAIN ? depth / 100 : depth;
            return true;
        }
        if (opcode.substr(0, name.size()) != name)
            continue;
        auto suffix = opcode.substr(name.size());
        const int field = ccField(suffix);
        if (field < 0)
            continue;
        if (target == CS_MOD_OFFSET && field == 1) {
            (void)integer(std::string(suffix), 0, 511);
            (void)integer(value, 0, 255);
            return true;                 // offset_curveccN has no effect in sfizz 1.2.3
        }
        if ((field == 2 && (envelopeShift || (target >= CS_MOD_ENV_DELAY && target <= CS_MOD_DELAY))) ||
            (field == 1 && target == CS_MOD_DELAY))
            return false;
        Modulation& m = binding(region.modulation, target, controllerNumber(suffix));
        if (field == 1) {
            m.curve = integer(value, 0, 255);
        } else if (field == 2) {
            m.smooth = integer(value, 0, 10000);
        } else {
            const bool percent = target == CS_MOD_AMPLITUDE || target == CS_MOD_PAN || target == CS_MOD_WIDTH ||
                target == CS_MOD_POSITION || baseTarget == CS_MOD_ENV_SUSTAIN || baseTarget == CS_MOD_ENV_START;
            m.depth = number(value, -1e9f, 1e9f) / (percent ? 100 : 1);
        }
        if (target >= CS_MOD_CUTOFF && target <= CS_MOD_FILTER_VELOCITY2) {
            const size_t slot = target == CS_MOD_CUTOFF2 || target == CS_MOD_RESONANCE2 || target == CS_MOD_FILTER_VELOCITY2;
            if (region.filters[slot].type == CS_FILTER_NONE)
                region.filters[slot].type = CS_FILTER_LOW2;
        }
        if (target >= CS_MOD_EQ1_FREQUENCY)
            region.eq[size_t((target - CS_MOD_EQ1_FREQUENCY) / 3)].enabled = true;
        return true;
    }
    return false;
}

// fileg_* and pitcheg_* (src/sfz/instrument.cpp:203-247).
bool envelopeOpcode(Region& region, const std::string& op, const std::string& value)
{
    std::string_view name(op);
    int slot;
    if (name.substr(0, 6) == "fileg_") { slot = 0; name.remove_prefix(6); }
    else if (name.substr(0, 8) == "pitcheg_") { slot = 1; name.remove_prefix(8); }
    else return false;
    auto& env = region.secondary[size_t(slot)];
    env.enabled = true;
    if (name == "depth") env.depth = number(value, -12000, 12000);
    else if (name == "vel2depth" || name == "veltodepth") env.velocityDepth = number(value, -12000, 12000);
    else if (name == "dynamic") env.dynamic = onOff(value);
    else if ((slot == 0 && name.substr(0, 7) == "depthcc") || (slot == 1 && name == "decay_shape")) {
        return true;                     // spellings sfizz 1.2.3 does not know
    } else if (name.substr(0, 10) == "depth_oncc" || name.substr(0, 13) == "depth_curvecc") {
        const bool curve = name.substr(0, 13) == "depth_curvecc";
        const int cc = controllerNumber(name.substr(curve ? 13 : 10));
        Modulation& m = binding(region.modulation, slot == 0 ? CS_MOD_FILEG_DEPTH : CS_MOD_PITCHEG_DEPTH, cc);
        if (curve) m.curve = integer(value, 0, 255);
        else m.depth = number(value, -12000, 12000);
    } else {
        constexpr std::string_view stages[] = {"delay", "attack", "hold", "decay", "sustain", "start", "release"};
        const auto found = std::find(std::begin(stages), std::end(stages), name);
        if (found != std::end(stages)) {
            const bool percent = name == "sustain" || name == "start";
            env.values[size_t(found - std::begin(stages))] = number(value, 0, 100) / (percent ? 100 : 1);
        } else {
            const int start = slot == 0 ? CS_MOD_FILEG_DELAY : CS_MOD_PITCHEG_DELAY;
            return modulationOpcode(region, "ampeg_" + std::string(name), value, start - CS_MOD_ENV_DELAY,
                                    &env.velocity);
        }
    }
    return true;
}

// lfoN_*, pitchlfo_*, amplfo_*, fillfo_* (src/sfz/instrument.cpp:249-327).
bool lfoOpcode(Region& region, const std::string& op, const std::string& value)
{
    std::string_view suffix(op);
    int index = 0;
    int legacy = CS_MOD_PITCH;
    if (suffix.substr(0, 3) == "lfo") {
        suffix.remove_prefix(3);
        const auto end = suffix.find('_');
        if (end == suffix.npos)
            return false;
        index = integer(std::string(suffix.substr(0, end)), 1, 64);
        suffix.remove_prefix(end + 1);
    } else if (suffix.substr(0, 9) == "pitchlfo_") {
        index = -1;
        suffix.remove_prefix(9);
    } else if (suffix.substr(0, 7) == "amplfo_") {
        index = -2;
        legacy = CS_MOD_VOLUME;
        suffix.remove_prefix(7);
    } else if (suffix.substr(0, 7) == "fillfo_") {
        index = -3;
        legacy = CS_MOD_CUTOFF;
        suffix.remove_prefix(7);
    } else {
        return false;
    }
    if (suffix.substr(0, 8) == "freq_lfo" && suffix.find("_oncc") != suffix.npos)
        return true;                     // unknown to sfizz 1.2.3
    Lfo& lfo = region.lfos[index];
    if (suffix == "wave" || suffix == "wave1") {
        const int wave = integer(value, -1, 12);
        if (wave >= 8 && wave < 12)
            throw std::runtime_error("unsupported LFO waveform " + value);
        lfo.wave = std::max(0, wave);
        return true;
    }
    static const std::pair<std::string_view, int> parameters[] = {
        {"freq", CS_MOD_LFO_FREQUENCY}, {"phase", CS_MOD_LFO_PHASE},
        {"delay", CS_MOD_LFO_DELAY}, {"fade", CS_MOD_LFO_FADE},
        {"pitch", CS_MOD_PITCH}, {"volume", CS_MOD_VOLUME}, {"pan", CS_MOD_PAN},
        {"width", CS_MOD_WIDTH}, {"position", CS_MOD_POSITION},
        {"cutoff2", CS_MOD_CUTOFF2}, {"cutoff1", CS_MOD_CUTOFF}, {"cutoff", CS_MOD_CUTOFF},
        {"resonance2", CS_MOD_RESONANCE2}, {"resonance1", CS_MOD_RESONANCE}, {"resonance", CS_MOD_RESONANCE},
        {"eq1freq", CS_MOD_EQ1_FREQUENCY}, {"eq1bw", CS_MOD_EQ1_BANDWIDTH}, {"eq1gain", CS_MOD_EQ1_GAIN},
        {"eq2freq", CS_MOD_EQ2_FREQUENCY}, {"eq2bw", CS_MOD_EQ2_BANDWIDTH}, {"eq2gain", CS_MOD_EQ2_GAIN},
        {"eq3freq", CS_MOD_EQ3_FREQUENCY}, {"eq3bw", CS_MOD_EQ3_BANDWIDTH}, {"eq3gain", CS_MOD_EQ3_GAIN},
    };
    const auto assign = [&](std::string_view field, int target) {
        const float unit = target == CS_MOD_PAN || target == CS_MOD_WIDTH || target == CS_MOD_POSITION ? 100.f : 1.f;
        if (field.empty()) {
            const float parsed = number(value, -24000, 24000) / unit;
            if (target == CS_MOD_LFO_FREQUENCY) lfo.frequency = parsed;
            else if (target == CS_MOD_LFO_PHASE) lfo.phase = parsed;
            else if (target == CS_MOD_LFO_DELAY) lfo.delay = parsed;
            else if (target == CS_MOD_LFO_FADE) lfo.fade = parsed;
            else lfo.depths[target] = parsed;
            return true;
        }
        const int kind = ccField(field);
        if (kind < 0)
            return false;
        Modulation& m = binding(lfo.modulation, target, controllerNumber(field));
        if (kind == 1) m.curve = integer(value, 0, 255);
        else if (kind == 2) m.smooth = integer(value, 0, 10000);
        else m.depth = number(value, -24000, 24000) / unit;
        return true;
    };
    if (index < 0 && suffix.substr(0, 5) == "depth")
        return assign(suffix.substr(5), legacy);
    for (const auto& [name, target] : parameters)
        if (suffix.substr(0, name.size()) == name && assign(suffix.substr(name.size()), target))
            return true;
    return false;
}

bool equalizerOpcode(Region& region, const std::string& op, const std::string& value)
{
    if (op.size() < 5 || op.compare(0, 2, "eq") != 0 || op[2] < '1' || op[2] > '3' || op[3] != '_')
        return false;
    Equalizer& eq = region.eq[size_t(op[2] - '1')];
    const auto field = std::string_view(op).substr(4);
    if (field == "freq") eq.frequency = number(value, 0, 20000);
    else if (field == "gain") eq.gain = number(value, -96, 96);
    else if (field == "bw") eq.bandwidth = number(value, .001f, 12);
    else return false;
    eq.enabled = true;
    return true;
}

// egN_* flexible envelopes driving pitch (src/sfz/instrument.cpp:343-367).
bool flexOpcode(Region& region, const std::string& op, const std::string& value)
{
    if (op.compare(0, 2, "eg") != 0 || op.size() < 5 || op[2] < '0' || op[2] > '9')
        return false;
    const auto separator = op.find('_', 2);
    if (separator == op.npos)
        return false;
    const int id = integer(op.substr(2, separator - 2), 1, 64);
    PitchEnvelope& env = region.pitchEnvelopes[id];
    auto field = std::string_view(op).substr(separator + 1);
    if (field == "sustain") env.sustain = integer(value, 0, 63);
    else if (field == "pitch") env.depth = number(value, -12000, 12000);
    else if (field.substr(0, 10) == "pitch_oncc") env.depthCC[controllerNumber(field.substr(10))] = number(value, -12000, 12000);
    else if (field.substr(0, 5) == "level") env.points[integer(std::string(field.substr(5)), 0, 63)].level = number(value, -1, 1);
    else if (field.substr(0, 4) == "time") {
        field.remove_prefix(4);
        const auto cc = field.find("_oncc");
        FlexPoint& point = env.points[integer(std::string(field.substr(0, cc)), 0, 63)];
        if (cc == field.npos) point.seconds = number(value, 0, 100);
        else point.timeCC[controllerNumber(field.substr(cc + 5))] = number(value, -100, 100);
    } else return false;
    return true;
}

bool filterOpcode(Region& region, const std::string& op, const std::string& value)
{
    std::string name = op;
    size_t slot = 0;
    if (name.compare(0, 5, "fil2_") == 0) { name.erase(3, 1); slot = 1; }
    else if (name.compare(0, 5, "fil1_") == 0) { name.erase(3, 1); }
    else if (name == "cutoff2" || name == "resonance2") { name.pop_back(); slot = 1; }
    else if (name == "cutoff1" || name == "resonance1") { name.pop_back(); }
    Filter& f = region.filters[slot];
    if (name == "cutoff") f.cutoff = number(value, 0, 20000);
    else if (name == "resonance") f.resonance = number(value, -60, 96);
    else if (name == "fil_keytrack") f.keyTrack = number(value, -12000, 12000);
    else if (name == "fil_keycenter") f.keyCenter = noteNumber(value);
    else if (name == "fil_veltrack") f.velocityTrack = number(value, -12000, 12000);
    else if (name == "fil_random" || name == "cutoff_random") f.random = number(value, -12000, 12000);
    else if (name == "fil_type") {
        static const std::map<std::string, int> types{
            {"lpf_1p", CS_FILTER_LOW1}, {"hpf_1p", CS_FILTER_HIGH1},
            {"lpf_2p", CS_FILTER_LOW2}, {"hpf_2p", CS_FILTER_HIGH2},
            {"bpf_2p", CS_FILTER_BAND2}, {"brf_2p", CS_FILTER_NOTCH2},
            {"lpf_4p", CS_FILTER_LOW4}, {"hpf_4p", CS_FILTER_HIGH4}, {"bpf_4p", CS_FILTER_BAND4},
            {"lpf_6p", CS_FILTER_LOW6}, {"hpf_6p", CS_FILTER_HIGH6}, {"bpf_6p", CS_FILTER_BAND6},
        };
        const auto type = types.find(value);
        if (type == types.end())
            throw std::runtime_error("unsupported filter type " + value);
        f.type = type->second;
    } else {
        return false;
    }
    if (f.type == CS_FILTER_NONE)
        f.type = CS_FILTER_LOW2;
    return true;
}

bool controllerFadeOpcode(Region& region, const std::string& op, const std::string& value)
{
    if (op == "xf_cccurve") {
        region.powerControllerFade = powerCurve(value);
        return true;
    }
    static const std::pair<std::string_view, int Crossfade::*> fields[] = {
        {"xfin_locc", &Crossfade::inLow}, {"xfin_hicc", &Crossfade::inHigh},
        {"xfout_locc", &Crossfade::outLow}, {"xfout_hicc", &Crossfade::outHigh},
    };
    for (const auto& [prefix, member] : fields) {
        if (std::string_view(op).substr(0, prefix.size()) != prefix)
            continue;
        const int cc = integer(op.substr(prefix.size()), 0, 127);
        region.controllerFades[cc].*member = integer(value, 0, 127);
        return true;
    }
    return false;
}

bool ignoredVariable(const std::string& op)
{
    if (op.compare(0, 3, "var") != 0)
        return false;
    const auto first = op.find_first_not_of("0123456789", 3);
    if (first == 3 || first == op.npos || op[first] != '_')
        return false;
    const std::string_view target(op.data() + first + 1, op.size() - first - 1);
    return target == "cutoff" || target == "mod" || target.substr(0, 4) == "oncc" ||
        target.substr(0, 7) == "curvecc" || target.substr(0, 2) == "eq";
}

void applyOpcode(Region& r, std::string& sample, std::map<int, Condition>& conditions,
                 std::map<int, Condition>& triggers, const std::string& op, const std::string& v)
{
    if (op == "sample") sample = v;
    else if (op == "key" || op == "group_label" || op == "master_label" || op == "global_label" ||
             op == "region_label" || op == "sw_label") return;
    else if (op == "lokey") r.lowKey = v == "-1" ? 0 : noteNumber(v);
    else if (op == "hikey") {
        r.triggerOnNote = v != "-1";
        r.highKey = r.triggerOnNote ? noteNumber(v) : 127;
    }
    else if (op == "pitch_keycenter") r.rootKey = noteNumber(v);
    else if (op == "lovel") r.lowVelocity = integer(v, 0, 127);
    else if (op == "hivel") r.highVelocity = integer(v, 0, 127);
    else if (op == "lochan" || op == "hichan") { (void)integer(v, 1, 16); }
    else if (op == "volume") r.volume += number(v, -144, 60);
    else if (op == "amplitude") r.amplitude *= number(v, 0, 10000) / 100;
    else if (op == "amp_veltrack") r.velocityTrack = number(v, -100, 100) / 100;
    else if (op == "amp_random") r.ampRandom = number(v, -24, 24);
    else if (op == "pitch_random") r.pitchRandom = number(v, -12000, 12000);
    else if (op.compare(0, 13, "amp_velcurve_") == 0) {
        const int velocity = integer(op.substr(13), 0, 127);
        const float value = number(v, 0, 1);
        const auto point = std::find_if(r.velocityCurve.begin(), r.velocityCurve.end(),
                                        [&](const auto& p) { return p.first == velocity; });
        if (point == r.velocityCurve.end()) r.velocityCurve.emplace_back(velocity, value);
        else point->second = value;
    }
    else if (op == "pan") r.pan = number(v, -100, 100) / 100;
    else if (op == "width") r.width = number(v, -100, 100) / 100;
    else if (op == "position") r.position = number(v, -100, 100) / 100;
    else if (op == "xfin_lokey") r.keyFade.inLow = noteNumber(v);
    else if (op == "xfin_hikey") r.keyFade.inHigh = noteNumber(v);
    else if (op == "xfout_lokey") r.keyFade.outLow = noteNumber(v);
    else if (op == "xfout_hikey") r.keyFade.outHigh = noteNumber(v);
    else if (op == "xfin_lovel") r.velocityFade.inLow = integer(v, 0, 127);
    else if (op == "xfin_hivel") r.velocityFade.inHigh = integer(v, 0, 127);
    else if (op == "xfout_lovel") r.velocityFade.outLow = integer(v, 0, 127);
    else if (op == "xfout_hivel") r.velocityFade.outHigh = integer(v, 0, 127);
    else if (op == "xf_keycurve") r.keyFade.power = powerCurve(v);
    else if (op == "xf_velcurve") r.velocityFade.power = powerCurve(v);
    else if (op == "tune" || op == "pitch") r.tune = number(v, -1200, 1200);
    else if (op == "transpose") r.transpose = integer(v, -127, 127);
    else if (op == "pitch_keytrack") r.keyTrack = number(v, -1200, 1200);
    else if (op == "bend_up" || op == "bendup") r.bendUp = number(v, -12000, 12000);
    else if (op == "bend_down" || op == "benddown") r.bendDown = number(v, -12000, 12000);
    else if (op == "bend_smooth") r.bendSmooth = integer(v, 0, 10000);
    else if (op == "delay") r.delay = number(v, 0, 100);
    else if (op == "group") r.group = integer64(v, -INT32_MAX, UINT32_MAX);
    else if (op == "note_polyphony") r.notePolyphony = integer(v, 1, 256);
    else if (op == "note_selfmask") r.selfMask = v == "mask" || onOff(v);
    else if (op == "oscillator_phase") r.oscillatorPhase = number(v, -1000, 1000);
    else if (op == "off_by" || op == "offby") {
        r.offBy = integer64(v, -INT32_MAX, UINT32_MAX);
        r.chokedByGroup = true;
    } else if (op == "off_mode" || op == "offmode") {
        if (v == "fast") r.offMode = OffMode::fast;
        else if (v == "normal") r.offMode = OffMode::normal;
        else if (v == "time") r.offMode = OffMode::time;
        else throw std::runtime_error("unsupported off mode " + v);
    } else if (op == "off_time") {
        r.offTime = number(v, 0, 100);
        r.offMode = OffMode::time;
    }
    else if (op == "offset") r.offset = integer(v, 0, INT32_MAX - 1);
    else if (op == "offset_random") r.offsetRandom = integer(v, 0, INT32_MAX - 1);
    else if (op == "end") r.end = integer(v, 0, INT32_MAX - 1);
    else if (op == "loop_start" || op == "loopstart") r.loopStart = integer(v, 0, INT32_MAX - 1);
    else if (op == "loop_end" || op == "loopend") r.loopEnd = integer(v, 0, INT32_MAX - 1);
    else if (op == "loop_crossfade") r.loopCrossfade = std::max(.001f, number(v, 0, 100));
    else if (op == "loop_type" || op == "looptype") {
        if (v != "forward" && v != "alternate" && v != "backward")
            throw std::runtime_error("unknown loop direction hint " + v);
    }
    else if (op == "ampeg_delay") r.envelopeDelay = number(v, 0, 100);
    else if (op == "ampeg_attack") r.attack = number(v, 0, 100);
    else if (op == "ampeg_hold") r.hold = number(v, 0, 100);
    else if (op == "ampeg_decay") r.decay = number(v, 0, 100);
    else if (op == "ampeg_sustain") r.sustain = number(v, 0, 100) / 100;
    else if (op == "ampeg_start") r.start = number(v, 0, 100) / 100;
    else if (op == "ampeg_release") r.release = number(v, 0, 100);
    else if (op == "ampeg_dynamic") r.envelopeDynamic = onOff(v);
    else if (op == "rt_decay") r.releaseDecay = number(v, 0, 200);
    else if (op == "rt_dead") r.releaseDead = onOff(v);
    else if (op == "sustain_sw") r.sustainEnabled = onOff(v);
    else if (op == "sustain_cc") r.sustainCC = integer(v, 0, 127);
    else if (op == "sustain_lo") r.sustainLow = integer(v, 0, 127);
    else if (op == "seq_length") r.sequenceLength = integer(v, 1, 1000000);
    else if (op == "seq_position") {
        r.sequencePosition = integer(v, 1, 1000000);
        r.explicitSequencePosition = true;
    }
    else if (op == "sw_default") r.switchDefault = noteNumber(v);
    else if (op == "sw_down") r.switchDown = noteNumber(v);
    else if (op == "sw_up") r.switchUp = noteNumber(v);
    else if (op == "sw_previous") r.switchPrevious = noteNumber(v);
    else if (op == "sw_lokey" || op == "sw_hikey") { (void)noteNumber(v); }
    else if (op == "sw_last") {
        if (!r.switchRange) r.switchLow = r.switchHigh = noteNumber(v);
    } else if (op == "sw_lolast" || op == "sw_hilast") {
        const int note = noteNumber(v);
        if (!r.switchRange) r.switchLow = r.switchHigh = note;
        (op == "sw_lolast" ? r.switchLow : r.switchHigh) = note;
        r.switchRange = true;
    }
    else if (op == "lorand") r.randomLow = number(v, 0, 1);
    else if (op == "hirand") r.randomHigh = number(v, 0, 1);
    else if (op == "trigger") {
        static const std::map<std::string, Trigger> values{{"attack", Trigger::attack}, {"release", Trigger::release},
            {"release_key", Trigger::releaseKey}, {"first", Trigger::first}, {"legato", Trigger::legato}};
        r.trigger = values.at(v);
    } else if (op == "loop_mode") {
        static const std::map<std::string, LoopMode> values{{"no_loop", LoopMode::none},
            {"one_shot", LoopMode::oneShot}, {"loop_continuous", LoopMode::continuous},
            {"loop_sustain", LoopMode::sustain}};
        r.loop = values.at(v);
    } else {
        if (modulationOpcode(r, op, v) || filterOpcode(r, op, v) || equalizerOpcode(r, op, v) || lfoOpcode(r, op, v) ||
            envelopeOpcode(r, op, v) || flexOpcode(r, op, v) || controllerFadeOpcode(r, op, v) ||
            ignoredVariable(op) || op == "ampeg_attack_shape" || op == "ampeg_release_shape")
            return;
        const bool trigger = op.compare(0, 3, "on_") == 0;
        const size_t skip = trigger ? 3 : 0;
        if (op.compare(skip, 4, "locc") != 0 && op.compare(skip, 4, "hicc") != 0)
            throw std::runtime_error("unsupported SFZ opcode");
        const auto cc = static_cast<uint8_t>(integer(op.substr(skip + 4), 0, 127));
        auto& ranges = trigger ? triggers : conditions;
        Condition& condition = ranges.emplace(cc, Condition{cc, 0, 127}).first->second;
        (op[skip] == 'l' ? condition.low : condition.high) = static_cast<uint8_t>(integer(v, 0, 127));
    }
}

class Loader {
public:
    Loader(Path root, SampleBank& bank) : root_(std::move(root)), bank_(bank) {}

    Instrument load(const Path& path)
    {
        parseFile(path, 0);
        if (current_ == "curve") flushCurve();
        else flushRegion();
        if (instrument_.regions.empty())
            throw std::runtime_error("no playable SFZ regions in " + path.u8string());
        return std::move(instrument_);
    }

private:
    void parseFile(const Path& file, int depth)
    {
        if (depth >= 32)
            throw std::runtime_error("too many nested SFZ includes");
        std::ifstream input(file, std::ios::binary);
        if (!input)
            throw std::runtime_error("cannot open SFZ " + file.u8string());
        const std::string text{std::istreambuf_iterator<char>(input), {}};
        const std::string_view src(text);
        size_t pos = src.substr(0, 3) == "\xef\xbb\xbf" ? 3 : 0;
        try {
            while (pos < src.size()) {
                pos = src.find_first_not_of(spaces, pos);
                if (pos == src.npos)
                    break;
                if (src.substr(pos, 2) == "//") {
                    pos = src.find('\n', pos);
                } else if (src[pos] == '<') {
                    const auto end = src.find('>', pos + 1);
                    if (end == src.npos)
                        throw std::runtime_error("unclosed SFZ header");
                    header(trimmed(src.substr(pos + 1, end - pos - 1)));
                    pos = end + 1;
                } else if (src[pos] == '#') {
                    const auto end = src.find('\n', pos);
                    const auto directive = src.substr(pos, end - pos);
                    if (directive.substr(0, 8) == "#include") {
                        const auto name = trimmed(directive.substr(8));
                        if (name.size() < 2 || name.front() != '"' || name.back() != '"')
                            throw std::runtime_error("expected quoted #include path");
                        parseFile(file.parent_path() / pathOf(unquoted(expand(name))), depth + 1);
                    } else if (directive.substr(0, 7) == "#define") {
                        const auto definition = trimmed(directive.substr(7));
                        const auto split = definition.find_first_of(spaces);
                        if (definition.empty() || definition.front() != '$' || split == definition.npos)
                            throw std::runtime_error("invalid #define");
                        macros_[definition.substr(0, split)] = expand(trimmed(definition.substr(split)));
                    } else {
                        throw std::runtime_error("unsupported SFZ directive " + std::string(directive));
                    }
                    pos = end;
                } else {
                    size_t end = pos;
                    while (end < src.size() && (nameChar(src[end]) || src[end] == '$'))
                        ++end;
                    const auto equals = src.find_first_not_of(" \t", end);
                    if (end == pos || equals == src.npos || src[equals] != '=')
                        throw std::runtime_error("expected opcode=value");
                    const auto name = expand(std::string(src.substr(pos, end - pos)));
                    pos = equals + 1;
                    bool quoted = false;
                    while (pos < src.size()) {
                        const char c = src[pos];
                        if (c == '"')
                            quoted = !quoted;
                        if (!quoted && (c == '\r' || c == '\n' || c == '<' || src.substr(pos, 2) == "//"))
                            break;
                        if (!quoted && (c == ' ' || c == '\t')) {
                            // A value ends where the next `name=` begins.
                            const auto next = src.find_first_not_of(" \t", pos);
                            auto tail = next;
                            while (tail < src.size() && (nameChar(src[tail]) || src[tail] == '$'))
                                ++tail;
                            const auto sep = src.find_first_not_of(" \t", tail);
                            if (tail != next && sep < src.size() && src[sep] == '=')
                                break;
                        }
                        ++pos;
                    }
                    if (quoted)
                        throw std::runtime_error("unclosed quoted value for " + name);
                    opcode(name, unquoted(expand(trimmed(src.substr(equals + 1, pos - equals - 1)))));
                }
            }
        } catch (const std::exception& error) {
            const auto line = 1 + std::count(src.begin(), src.begin() + std::min(pos, src.size()), '\n');
            throw std::runtime_error(file.u8string() + ":" + std::to_string(line) + ": " + error.what());
        }
    }

    std::string expand(std::string value) const
    {
        size_t pos = 0;
        while ((pos = value.find('$', pos)) != value.npos) {
            size_t end = pos + 1;
            while (end < value.size() && nameChar(value[end]))
                ++end;
            const auto name = value.substr(pos, end - pos);
            const auto it = macros_.find(name);
            if (it == macros_.end())
                throw std::runtime_error("undefined SFZ macro " + name);
            value.replace(pos, end - pos, it->second);
            pos += it->second.size();
        }
        return value;
    }

    void header(const std::string& name)
    {
        if (current_ == "curve") flushCurve();
        else flushRegion();
        current_ = name;
        if (name == "global") {
            global_.clear();
            master_.clear();
            group_.clear();
        } else if (name == "master") {
            master_.clear();
            group_.clear();
        } else if (name == "group") {
            group_.clear();
        } else if (name != "region" && name != "control" && name != "curve") {
            throw std::runtime_error("unsupported SFZ header <" + name + ">");
        }
    }

    void opcode(const std::string& name, const std::string& value)
    {
        if (value.empty())
            throw std::runtime_error("empty value for " + name);
        if (current_ == "global") global_[name] = value;
        else if (current_ == "master") master_[name] = value;
        else if (current_ == "group") group_[name] = value;
        else if (current_ == "region") region_[name] = value;
        else if (current_ == "curve") curve_[name] = value;
        else if (current_ == "control") control(name, value);
        else throw std::runtime_error("opcode outside SFZ header " + name);
    }

    void control(const std::string& name, const std::string& value)
    {
        if (name == "default_path") {
            defaultPath_ = pathOf(value);
        } else if (name.compare(0, 6, "set_cc") == 0) {
            const int cc = integer(name.substr(6), 0, 511);
            const float raw = number(value, 0, 127);
            if (cc < 128) instrument_.initialCC[size_t(cc)] = raw;
            else instrument_.extendedCCDefaults[cc] = raw;
        } else if (name.compare(0, 8, "set_hdcc") == 0) {
            const int cc = integer(name.substr(8), 0, 511);
            const float raw = 127 * number(value, 0, 1);
            if (cc < 128) instrument_.initialCC[size_t(cc)] = raw;
            else instrument_.extendedCCDefaults[cc] = raw;
        } else if (name.compare(0, 8, "label_cc") == 0) {
            (void)integer(name.substr(8), 0, 511);
        } else if (name.compare(0, 9, "label_key") == 0) {
            (void)integer(name.substr(9), 0, 127);
        } else if (name != "image" && name != "image_controls") {
            throw std::runtime_error("unsupported control opcode " + name);
        }
    }

    void flushCurve()
    {
        const auto index = curve_.find("curve_index");
        if (index == curve_.end() && explicitCurves_) {
            curve_.clear();
            return;
        }
        const int id = index == curve_.end() ? nextCurve_++ : integer(index->second, 0, 255);
        explicitCurves_ |= index != curve_.end();
        std::map<int, float> points{{0, 0}, {127, 1}};
        for (const auto& [key, value] : curve_) {
            if (key == "curve_index")
                continue;
            if (key.front() != 'v')
                throw std::runtime_error("unsupported <curve> opcode " + key);
            points[integer(key.substr(1), 0, 127)] = number(value, -1e16f, 1e16f);
        }
        Curve& curve = instrument_.curves[id];
        for (auto lo = points.begin(), hi = std::next(lo); hi != points.end(); ++lo, ++hi) {
            for (int x = lo->first; x <= hi->first; ++x) {
                const float phase = float(x - lo->first) / (hi->first - lo->first);
                curve[size_t(x)] = std::clamp(lo->second + phase * (hi->second - lo->second), -1.f, 1.f);
            }
        }
        curve_.clear();
    }

    void flushRegion()
    {
        if (current_ != "region")
            return;
        Region region;
        std::string sample;
        std::map<int, Condition> conditions, triggers;
        for (const auto* scope : {&global_, &master_, &group_, &region_}) {
            // `key` sets all three key fields; specific fields in the same scope win.
            if (const auto it = scope->find("key"); it != scope->end()) {
                region.triggerOnNote = it->second != "-1";
                region.lowKey = region.highKey = region.rootKey = region.triggerOnNote ? noteNumber(it->second) : 60;
            }
            for (const auto& [op, value] : *scope) {
                try {
                    applyOpcode(region, sample, conditions, triggers, op, value);
                } catch (const std::exception& error) {
                    throw std::runtime_error(op + "=" + value + ": " + error.what());
                }
            }
        }
        const bool emptyBlock = region_.empty();
        region_.clear();
        if (sample.empty() && emptyBlock)
            sample = "*silence";
        if (sample == "*sine") region.generator = CS_GEN_SINE;
        else if (sample == "*silence") region.generator = CS_GEN_SILENCE;
        else if (sample == "*noise") region.generator = CS_GEN_NOISE;
        else if (sample.empty() || sample.front() == '*')
            throw std::runtime_error("missing or unsupported region sample " + sample);
        if ((region.lowKey > region.highKey && triggers.empty()) || region.lowVelocity > region.highVelocity ||
            region.randomLow > region.randomHigh || region.switchLow > region.switchHigh)
            throw std::runtime_error("invalid region range for " + sample);
        if (!region.velocityCurve.empty()) {
            std::sort(region.velocityCurve.begin(), region.velocityCurve.end());
            if (region.velocityCurve.front().first != 0)
                region.velocityCurve.insert(region.velocityCurve.begin(), {0, 0});
            if (region.velocityCurve.back().first != 127)
                region.velocityCurve.emplace_back(127, 1);
        }
        if (region.generator == CS_GEN_NONE) {
            region.sample = bank_.describe((root_ / defaultPath_ / pathOf(sample)).string());
            const Sample& audio = bank_.samples[size_t(region.sample)];
            region.end = region.end < 0 ? audio.frames : std::min(region.end + 1, audio.frames);
            if (region.offset >= region.end)
                throw std::runtime_error("offset past end of sample " + sample);
            if (region.loop == LoopMode::automatic)
                region.loop = audio.loopEnd > 0 || region.loopEnd >= 0 ? LoopMode::continuous : LoopMode::none;
            if (region.loop == LoopMode::continuous || region.loop == LoopMode::sustain) {
                if (region.loopStart < 0) region.loopStart = audio.loopFirst;
                if (region.loopEnd < 0) region.loopEnd = audio.loopEnd > 0 ? audio.loopEnd : region.end;
                else region.loopEnd = std::min(region.loopEnd + 1, region.end);
                if (region.loopStart >= region.loopEnd || region.loopEnd > region.end || region.offset >= region.loopEnd)
                    throw std::runtime_error("invalid forward loop in " + sample);
            }
        }
        for (const auto& [cc, condition] : conditions) {
            if (condition.low > condition.high)
                throw std::runtime_error("invalid CC range for " + sample);
            region.conditions.push_back(condition);
            instrument_.usedCC[size_t(cc)] = true;
        }
        for (auto& [cc, fade] : region.controllerFades) {
            fade.power = region.powerControllerFade;
            instrument_.usedCC[size_t(cc)] = true;
        }
        for (const auto& m : region.modulation)
            if (m.cc < 128)
                instrument_.usedCC[size_t(m.cc)] = true;
        for (const auto& [index, lfo] : region.lfos) {
            (void)index;
            const auto enableFilter = [&](int target) {
                const size_t second = target == CS_MOD_CUTOFF2 || target == CS_MOD_RESONANCE2;
                if (target >= CS_MOD_CUTOFF && target <= CS_MOD_RESONANCE2 && region.filters[second].type == CS_FILTER_NONE)
                    region.filters[second].type = CS_FILTER_LOW2;
                if (target >= CS_MOD_EQ1_FREQUENCY)
                    region.eq[size_t((target - CS_MOD_EQ1_FREQUENCY) / 3)].enabled = true;
            };
            for (const auto& depth : lfo.depths)
                enableFilter(depth.first);
            for (const auto& m : lfo.modulation) {
                if (m.cc < 128)
                    instrument_.usedCC[size_t(m.cc)] = true;
                enableFilter(m.target);
            }
        }
        for (const auto& [id, env] : region.pitchEnvelopes) {
            (void)id;
            if (env.points.empty() || env.points.rbegin()->second.level != 0 ||
                (env.sustain >= 0 && env.sustain != env.points.rbegin()->first))
                throw std::runtime_error("flexible pitch envelope must end at a zero-level sustain point");
            for (const auto& cc : env.depthCC)
                if (cc.first < 128)
                    instrument_.usedCC[size_t(cc.first)] = true;
            for (const auto& point : env.points)
                for (const auto& cc : point.second.timeCC)
                    if (cc.first < 128)
                        instrument_.usedCC[size_t(cc.first)] = true;
        }
        if (region.sustainEnabled)
            instrument_.usedCC[size_t(region.sustainCC)] = true;
        const int index = int(instrument_.regions.size());
        if (region.triggerOnNote)
            for (int note = region.lowKey; note <= region.highKey; ++note)
                instrument_.byKey[size_t(note)].push_back(index);
        for (const auto& [cc, condition] : triggers) {
            if (condition.low > condition.high)
                throw std::runtime_error("invalid CC trigger range for " + sample);
            region.ccTriggers.push_back(condition);
            instrument_.byCC[size_t(cc)].push_back(index);
            instrument_.usedCC[size_t(cc)] = true;
        }
        if (region.switchLow >= 0)
            for (int note = region.switchLow; note <= region.switchHigh; ++note)
                instrument_.switchKeys[size_t(note)] = true;
        if (region.switchDefault >= 0)
            instrument_.initialSwitch = region.switchDefault;
        instrument_.hasOffBy |= region.chokedByGroup;
        instrument_.regions.push_back(std::move(region));
    }

    Path root_, defaultPath_;
    SampleBank& bank_;
    Instrument instrument_;
    std::string current_;
    Opcodes global_, master_, group_, region_, macros_, curve_;
    int nextCurve_ = 7;
    bool explicitCurves_ = false;
};

} // namespace

Instrument loadInstrument(const std::string& path, SampleBank& bank)
{
    const Path file = std::filesystem::u8path(path);
    return Loader(file.parent_path(), bank).load(file);
}

// Controller curves (src/sfz/instrument.cpp:909-931): a <curve> table, else the
// built-in curves 0-6, linearly interpolated between integer controller values.
float curveValue(const Instrument& instrument, int curve, float value)
{
    value = std::clamp(value, 0.f, 127.f);
    const int lo = static_cast<int>(value);
    const int hi = std::min(127, lo + 1);
    const float fraction = value - float(lo);
    if (const auto custom = instrument.curves.find(curve); custom != instrument.curves.end())
        return custom->second[size_t(lo)] + fraction * (custom->second[size_t(hi)] - custom->second[size_t(lo)]);
    const auto at = [curve](int key) {
        const float x = float(key) / 127.f;
        switch (curve) {
        case 1: return 2 * x - 1;
        case 2: return 1 - x;
        case 3: return 1 - 2 * x;
        case 4: return x * x;
        case 5: return std::sqrt(x);
        case 6: return std::sqrt(1 - x);
        default: return x;
        }
    };
    const float a = at(lo);
    return a + fraction * (at(hi) - a);
}

} // namespace csh
