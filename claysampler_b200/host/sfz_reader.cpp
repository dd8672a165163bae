// SFZ instruments: text -> scoped opcode tables -> regions of the host model.
//
// Reading happens in three layers.  The lexer walks the text (headers, opcodes,
// comments, #define / #include) and hands each `name=value` to the current
// scope.  When a <region> closes, its effective opcodes (<global>, <master>,
// <group>, <region>, each applied in opcode-name order, later scopes on top) go
// through a dispatcher: exact opcode names first, then opcode families matched by
// prefix (controller-bound parameters, filters, EQ bands, LFOs, the filter and
// pitch envelopes, flex envelopes, controller crossfades, CC ranges).  Last, the
// region is resolved against its sample (end, loop) and indexed by key and
// controller.  The accepted opcodes, their ranges, defaults and the order in which
// they apply are the SFZ format's as sfizz 1.2.3 reads it, which the reference
// follows (src/sfz/instrument.cpp); so are the error messages the command line
// prints.
#include "model.hpp"

#include <cctype>
#include <cmath>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iterator>
#include <stdexcept>
#include <string_view>
#include <unordered_map>

namespace clayhost {
namespace {

using Path = std::filesystem::path;
using Scope = std::map<std::string, std::string>;   // opcode name -> value, applied in name order
constexpr std::string_view kSpaces = " \t\r\n";

[[noreturn]] void fail(const std::string& message) { throw std::runtime_error(message); }

std::string stripped(std::string_view text)
{
    const auto a = text.find_first_not_of(kSpaces);
    if (a == text.npos)
        return {};
    return std::string(text.substr(a, text.find_last_not_of(kSpaces) - a + 1));
}

bool opcodeChar(char c) { return std::isalnum(static_cast<unsigned char>(c)) || c == '_'; }

bool startsWith(std::string_view text, std::string_view prefix) { return text.substr(0, prefix.size()) == prefix; }

std::string dequoted(const std::string& text)
{
    return text.size() >= 2 && text.front() == '"' && text.back() == '"' ? text.substr(1, text.size() - 2) : text;
}

Path portablePath(std::string text)
{
    for (char& c : text)
        if (c == '\\')
            c = '/';
    return std::filesystem::u8path(text);
}

// ---- values ----------------------------------------------------------------------

float real(const std::string& text, float lo, float hi)
{
    size_t used = 0;
    const float v = std::stof(text, &used);
    if (used != text.size() || !std::isfinite(v) || v < lo || v > hi)
        fail("invalid value " + text);
    return v;
}

int64_t whole64(const std::string& text, int64_t lo, int64_t hi)
{
    size_t used = 0;
    const long long v = std::stoll(text, &used);
    if (used != text.size() || v < lo || v > hi)
        fail("invalid value " + text);
    return v;
}

int whole(const std::string& text, int lo, int hi) { return static_cast<int>(whole64(text, lo, hi)); }

// A MIDI note: a number, or a name such as c4, F#3 or Bb-1 (middle C is c4 = 60).
int noteNumber(const std::string& text)
{
    const int letter = text.empty() ? 0 : std::toupper(static_cast<unsigned char>(text[0]));
    if (text.size() < 2 || letter < 'A' || letter > 'G')
        return whole(text, 0, 127);
    static constexpr int kPitchClass[] = {9, 11, 0, 2, 4, 5, 7};   // A B C D E F G
    int note = kPitchClass[letter - 'A'];
    size_t at = 1;
    if (text[at] == '#')
        ++note, ++at;
    else if (text[at] == 'b')
        --note, ++at;
    note += 12 * (whole(text.substr(at), -2, 10) + 1);
    if (note < 0 || note > 127)
        fail("key outside MIDI range " + text);
    return note;
}

bool onOff(const std::string& text)
{
    if (text == "on" || text == "1")
        return true;
    if (text == "off" || text == "0")
        return false;
    fail("invalid switch " + text);
}

bool powerCurve(const std::string& text)
{
    if (text == "power")
        return true;
    if (text == "gain")
        return false;
    fail("unsupported crossfade curve " + text);
}

// Controller numbers of modulation opcodes: 0-127 and the extended sources, but
// not 128-130, which the format reserves for sources this renderer lacks.
int modulationCc(std::string_view text)
{
    const int cc = whole(std::string(text), 0, 511);
    if (cc >= 128 && cc <= 130)
        fail("unsupported extended controller CC" + std::to_string(cc));
    return cc;
}

// ---- controller-bound parameters (<param>_oncc<N>, _cc<N>, cc<N>, _curvecc<N>, _smoothcc<N>) ----

enum class CcField { depth, curve, smooth };

// Splits "<suffix>" after a parameter name into the controller field and the
// controller text; false when the suffix is not a controller form.
bool ccSuffix(std::string_view rest, CcField& field, std::string_view& cc)
{
    static constexpr std::pair<std::string_view, CcField> kForms[] = {
        {"_oncc", CcField::depth}, {"_cc", CcField::depth}, {"cc", CcField::depth},
        {"_curvecc", CcField::curve}, {"_smoothcc", CcField::smooth},
    };
    for (const auto& [form, kind] : kForms)
        if (startsWith(rest, form)) {
            field = kind;
            cc = rest.substr(form.size());
            return true;
        }
    return false;
}

struct Parameter {
    std::string_view name;
    int target;
};

// Parameters a controller can drive, by opcode name.
constexpr Parameter kBindable[] = {
    {"amplitude", CS_MOD_AMPLITUDE}, {"volume", CS_MOD_VOLUME}, {"gain", CS_MOD_VOLUME},
    {"pan", CS_MOD_PAN}, {"width", CS_MOD_WIDTH}, {"position", CS_MOD_POSITION},
    {"pitch", CS_MOD_PITCH}, {"tune", CS_MOD_PITCH},
    {"ampeg_delay", CS_MOD_ENV_DELAY}, {"ampeg_attack", CS_MOD_ENV_ATTACK}, {"ampeg_hold", CS_MOD_ENV_HOLD},
    {"ampeg_decay", CS_MOD_ENV_DECAY}, {"ampeg_sustain", CS_MOD_ENV_SUSTAIN}, {"ampeg_start", CS_MOD_ENV_START},
    {"ampeg_release", CS_MOD_ENV_RELEASE}, {"offset", CS_MOD_OFFSET}, {"delay", CS_MOD_DELAY},
    {"cutoff", CS_MOD_CUTOFF}, {"cutoff1", CS_MOD_CUTOFF}, {"cutoff2", CS_MOD_CUTOFF2},
    {"resonance", CS_MOD_RESONANCE}, {"resonance1", CS_MOD_RESONANCE}, {"resonance2", CS_MOD_RESONANCE2},
    {"fil_veltrack", CS_MOD_FILTER_VELOCITY}, {"fil1_veltrack", CS_MOD_FILTER_VELOCITY},
    {"fil2_veltrack", CS_MOD_FILTER_VELOCITY2},
    {"eq1_freq", CS_MOD_EQ1_FREQUENCY}, {"eq1_bw", CS_MOD_EQ1_BANDWIDTH}, {"eq1_gain", CS_MOD_EQ1_GAIN},
    {"eq2_freq", CS_MOD_EQ2_FREQUENCY}, {"eq2_bw", CS_MOD_EQ2_BANDWIDTH}, {"eq2_gain", CS_MOD_EQ2_GAIN},
    {"eq3_freq", CS_MOD_EQ3_FREQUENCY}, {"eq3_bw", CS_MOD_EQ3_BANDWIDTH}, {"eq3_gain", CS_MOD_EQ3_GAIN},
};

bool isEnvelopeTarget(int target) { return target >= CS_MOD_ENV_DELAY && target <= CS_MOD_ENV_RELEASE; }

CcBinding& bindingFor(std::vector<CcBinding>& list, int target, int cc)
{
    for (CcBinding& b : list)
        if (b.target == target && b.cc == cc)
            return b;
    list.push_back({target, cc});
    return list.back();
}

// A filter slot or EQ band named by a modulation target is switched on (a
// modulated cutoff on an unfiltered region gets the default 2-pole low-pass).
void enableFor(Region& r, int target)
{
    if (target >= CS_MOD_CUTOFF && target <= CS_MOD_RESONANCE2) {
        const int slot = target == CS_MOD_CUTOFF2 || target == CS_MOD_RESONANCE2;
        if (r.filters[slot].type == CS_FILTER_NONE)
            r.filters[slot].type = CS_FILTER_LOW2;
    }
    if (target >= CS_MOD_EQ1_FREQUENCY)
        r.eqs[(target - CS_MOD_EQ1_FREQUENCY) / 3].on = true;
}

// ampeg_* controller and velocity forms; `shift` moves the envelope targets to
// the filter or pitch envelope's, whose velocity table is `velocity`.
bool bindable(Region& r, const std::string& op, const std::string& value, int shift = 0,
              std::array<float, kStages>* velocity = nullptr)
{
    // Velocity tracking of the envelope stages (ampeg_vel2<stage>, ampeg_velto<stage>).
    static constexpr std::pair<std::string_view, int> kVelocityStages[] = {
        {"delay", kDelay}, {"attack", kAttack}, {"hold", kHold}, {"decay", kDecay}, {"sustain", kSustain},
        {"release", kRelease},
    };
    for (const std::string_view form : {std::string_view("ampeg_vel2"), std::string_view("ampeg_velto")}) {
        if (!startsWith(op, form))
            continue;
        for (const auto& [stage, index] : kVelocityStages)
            if (std::string_view(op).substr(form.size()) == stage) {
                const float depth = real(value, -100, 100);
                (velocity ? *velocity : r.ampEnvelope.perVelocity)[size_t(index)] =
                    index == kSustain ? depth / 100 : depth;
                return true;
            }
    }
    for (const Parameter& p : kBindable) {
        if (shift && !isEnvelopeTarget(p.target))
            continue;
        if (!startsWith(op, p.name))
            continue;
        CcField field;
        std::string_view ccText;
        if (!ccSuffix(std::string_view(op).substr(p.name.size()), field, ccText))
            continue;
        const int target = p.target + shift;
        if (target == CS_MOD_OFFSET && field == CcField::curve) {
            (void)whole(std::string(ccText), 0, 511);    // accepted and ignored, as sfizz 1.2.3 does
            (void)whole(value, 0, 255);
            return true;
        }
        const bool timing = target >= CS_MOD_ENV_DELAY && target <= CS_MOD_DELAY;
        if ((field == CcField::smooth && (shift || timing)) || (field == CcField::curve && target == CS_MOD_DELAY))
            return false;
        CcBinding& b = bindingFor(r.bindings, target, modulationCc(ccText));
        if (field == CcField::curve) {
            b.curve = whole(value, 0, 255);
        } else if (field == CcField::smooth) {
            b.smoothMs = whole(value, 0, 10000);
        } else {
            const bool percent = target == CS_MOD_AMPLITUDE || target == CS_MOD_PAN || target == CS_MOD_WIDTH ||
                target == CS_MOD_POSITION || p.target == CS_MOD_ENV_SUSTAIN || p.target == CS_MOD_ENV_START;
            b.depth = real(value, -1e9f, 1e9f) / (percent ? 100 : 1);
        }
        if (target >= CS_MOD_CUTOFF && target <= CS_MOD_FILTER_VELOCITY2) {
            const int slot = target == CS_MOD_CUTOFF2 || target == CS_MOD_RESONANCE2 || target == CS_MOD_FILTER_VELOCITY2;
            if (r.filters[slot].type == CS_FILTER_NONE)
                r.filters[slot].type = CS_FILTER_LOW2;
        }
        if (target >= CS_MOD_EQ1_FREQUENCY)
            r.eqs[(target - CS_MOD_EQ1_FREQUENCY) / 3].on = true;
        return true;
    }
    return false;
}

// ---- the filter and pitch envelopes (fileg_*, pitcheg_*) ------------------------------

bool auxEnvelope(Region& r, const std::string& op, const std::string& value)
{
    int slot;
    std::string_view rest(op);
    if (startsWith(rest, "fileg_")) {
        slot = 0;
        rest.remove_prefix(6);
    } else if (startsWith(rest, "pitcheg_")) {
        slot = 1;
        rest.remove_prefix(8);
    } else {
        return false;
    }
    AuxEnvelope& env = r.aux[size_t(slot)];
    env.on = true;
    if (rest == "depth") {
        env.depth = real(value, -12000, 12000);
    } else if (rest == "vel2depth" || rest == "veltodepth") {
        env.velocityDepth = real(value, -12000, 12000);
    } else if (rest == "dynamic") {
        env.shape.dynamic = onOff(value);
    } else if ((slot == 0 && startsWith(rest, "depthcc")) || (slot == 1 && rest == "decay_shape")) {
        return true;                    // spellings sfizz 1.2.3 does not know: accepted, no effect
    } else if (startsWith(rest, "depth_oncc") || startsWith(rest, "depth_curvecc")) {
        const bool curve = startsWith(rest, "depth_curvecc");
        const int cc = modulationCc(rest.substr(curve ? 13 : 10));
        CcBinding& b = bindingFor(r.bindings, slot == 0 ? CS_MOD_FILEG_DEPTH : CS_MOD_PITCHEG_DEPTH, cc);
        if (curve)
            b.curve = whole(value, 0, 255);
        else
            b.depth = real(value, -12000, 12000);
    } else {
        static constexpr std::pair<std::string_view, int> kStageNames[] = {
            {"delay", kDelay}, {"attack", kAttack}, {"hold", kHold}, {"decay", kDecay},
            {"sustain", kSustain}, {"start", kStart}, {"release", kRelease},
        };
        for (const auto& [name, index] : kStageNames)
            if (rest == name) {
                const bool level = index == kSustain || index == kStart;
                env.shape.stage[size_t(index)] = real(value, 0, 100) / (level ? 100 : 1);
                return true;
            }
        // Controller and velocity forms of the stages, on this envelope's targets.
        const int first = slot == 0 ? CS_MOD_FILEG_DELAY : CS_MOD_PITCHEG_DELAY;
        return bindable(r, "ampeg_" + std::string(rest), value, first - CS_MOD_ENV_DELAY, &env.shape.perVelocity);
    }
    return true;
}

// ---- LFOs (lfo<N>_*, and the legacy pitchlfo_, amplfo_, fillfo_ forms) -----------------

bool lfoOpcode(Region& r, const std::string& op, const std::string& value)
{
    std::string_view rest(op);
    int index;
    int legacyTarget = CS_MOD_PITCH;
    if (startsWith(rest, "lfo")) {
        rest.remove_prefix(3);
        const auto underscore = rest.find('_');
        if (underscore == rest.npos)
            return false;
        index = whole(std::string(rest.substr(0, underscore)), 1, 64);
        rest.remove_prefix(underscore + 1);
    } else if (startsWith(rest, "pitchlfo_")) {
        index = -1;
        rest.remove_prefix(9);
    } else if (startsWith(rest, "amplfo_")) {
        index = -2;
        legacyTarget = CS_MOD_VOLUME;
        rest.remove_prefix(7);
    } else if (startsWith(rest, "fillfo_")) {
        index = -3;
        legacyTarget = CS_MOD_CUTOFF;
        rest.remove_prefix(7);
    } else {
        return false;
    }
    if (startsWith(rest, "freq_lfo") && rest.find("_oncc") != rest.npos)
        return true;                    // LFO-to-LFO frequency controllers: unknown to sfizz 1.2.3
    LfoSpec& lfo = r.lfos.slot(index);
    if (rest == "wave" || rest == "wave1") {
        const int wave = whole(value, -1, 12);
        if (wave >= 8 && wave < 12)
            fail("unsupported LFO waveform " + value);
        lfo.wave = std::max(0, wave);
        return true;
    }
    // Assigns `field` (empty: the base value) of the LFO parameter `target`.
    const auto assign = [&](std::string_view field, int target) {
        const float unit = target == CS_MOD_PAN || target == CS_MOD_WIDTH || target == CS_MOD_POSITION ? 100.f : 1.f;
        if (field.empty()) {
            const float v = real(value, -24000, 24000) / unit;
            switch (target) {
            case CS_MOD_LFO_FREQUENCY: lfo.frequency = v; break;
            case CS_MOD_LFO_PHASE: lfo.phase = v; break;
            case CS_MOD_LFO_DELAY: lfo.delay = v; break;
            case CS_MOD_LFO_FADE: lfo.fade = v; break;
            default: lfo.depth.slot(target) = v; break;
            }
            return true;
        }
        CcField kind;
        std::string_view ccText;
        if (!ccSuffix(field, kind, ccText))
            return false;
        CcBinding& b = bindingFor(lfo.ccs, target, modulationCc(ccText));
        if (kind == CcField::curve)
            b.curve = whole(value, 0, 255);
        else if (kind == CcField::smooth)
            b.smoothMs = whole(value, 0, 10000);
        else
            b.depth = real(value, -24000, 24000) / unit;
        return true;
    };
    if (index < 0 && startsWith(rest, "depth"))
        return assign(rest.substr(5), legacyTarget);
    // Longer names before their prefixes (cutoff2 before cutoff).
    static constexpr Parameter kLfoParameters[] = {
        {"freq", CS_MOD_LFO_FREQUENCY}, {"phase", CS_MOD_LFO_PHASE}, {"delay", CS_MOD_LFO_DELAY},
        {"fade", CS_MOD_LFO_FADE}, {"pitch", CS_MOD_PITCH}, {"volume", CS_MOD_VOLUME}, {"pan", CS_MOD_PAN},
        {"width", CS_MOD_WIDTH}, {"position", CS_MOD_POSITION},
        {"cutoff2", CS_MOD_CUTOFF2}, {"cutoff1", CS_MOD_CUTOFF}, {"cutoff", CS_MOD_CUTOFF},
        {"resonance2", CS_MOD_RESONANCE2}, {"resonance1", CS_MOD_RESONANCE}, {"resonance", CS_MOD_RESONANCE},
        {"eq1freq", CS_MOD_EQ1_FREQUENCY}, {"eq1bw", CS_MOD_EQ1_BANDWIDTH}, {"eq1gain", CS_MOD_EQ1_GAIN},
        {"eq2freq", CS_MOD_EQ2_FREQUENCY}, {"eq2bw", CS_MOD_EQ2_BANDWIDTH}, {"eq2gain", CS_MOD_EQ2_GAIN},
        {"eq3freq", CS_MOD_EQ3_FREQUENCY}, {"eq3bw", CS_MOD_EQ3_BANDWIDTH}, {"eq3gain", CS_MOD_EQ3_GAIN},
    };
    for (const Parameter& p : kLfoParameters)
        if (startsWith(rest, p.name) && assign(rest.substr(p.name.size()), p.target))
            return true;
    return false;
}

// ---- EQ bands, filters, flex envelopes, controller crossfades ---------------------------

bool eqOpcode(Region& r, const std::string& op, const std::string& value)
{
    if (op.size() < 5 || op.compare(0, 2, "eq") != 0 || op[2] < '1' || op[2] > '3' || op[3] != '_')
        return false;
    EqSpec& eq = r.eqs[size_t(op[2] - '1')];
    const std::string_view field = std::string_view(op).substr(4);
    if (field == "freq") eq.frequency = real(value, 0, 20000);
    else if (field == "gain") eq.gain = real(value, -96, 96);
    else if (field == "bw") eq.bandwidth = real(value, .001f, 12);
    else return false;
    eq.on = true;
    return true;
}

bool filterOpcode(Region& r, const std::string& op, const std::string& value)
{
    // fil2_* / cutoff2 / resonance2 address the second filter; fil1_*, cutoff1 and
    // resonance1 are the first filter's long spellings.
    std::string name = op;
    size_t slot = 0;
    if (name.compare(0, 5, "fil2_") == 0) {
        name.erase(3, 1);
        slot = 1;
    } else if (name.compare(0, 5, "fil1_") == 0) {
        name.erase(3, 1);
    } else if (name == "cutoff2" || name == "resonance2") {
        name.pop_back();
        slot = 1;
    } else if (name == "cutoff1" || name == "resonance1") {
        name.pop_back();
    }
    FilterSpec& f = r.filters[slot];
    static const std::unordered_map<std::string, int> kTypes{
        {"lpf_1p", CS_FILTER_LOW1}, {"hpf_1p", CS_FILTER_HIGH1}, {"lpf_2p", CS_FILTER_LOW2},
        {"hpf_2p", CS_FILTER_HIGH2}, {"bpf_2p", CS_FILTER_BAND2}, {"brf_2p", CS_FILTER_NOTCH2},
        {"lpf_4p", CS_FILTER_LOW4}, {"hpf_4p", CS_FILTER_HIGH4}, {"bpf_4p", CS_FILTER_BAND4},
        {"lpf_6p", CS_FILTER_LOW6}, {"hpf_6p", CS_FILTER_HIGH6}, {"bpf_6p", CS_FILTER_BAND6},
    };
    if (name == "cutoff") f.cutoff = real(value, 0, 20000);
    else if (name == "resonance") f.resonance = real(value, -60, 96);
    else if (name == "fil_keytrack") f.keyTrack = real(value, -12000, 12000);
    else if (name == "fil_keycenter") f.keyCenter = noteNumber(value);
    else if (name == "fil_veltrack") f.velocityTrack = real(value, -12000, 12000);
    else if (name == "fil_random" || name == "cutoff_random") f.random = real(value, -12000, 12000);
    else if (name == "fil_type") {
        const auto type = kTypes.find(value);
        if (type == kTypes.end())
            fail("unsupported filter type " + value);
        f.type = type->second;
    } else {
        return false;
    }
    if (f.type == CS_FILTER_NONE)
        f.type = CS_FILTER_LOW2;
    return true;
}

bool flexOpcode(Region& r, const std::string& op, const std::string& value)
{
    if (op.compare(0, 2, "eg") != 0 || op.size() < 5 || op[2] < '0' || op[2] > '9')
        return false;
    const auto underscore = op.find('_', 2);
    if (underscore == op.npos)
        return false;
    FlexEnvelope& env = r.flex.slot(whole(op.substr(2, underscore - 2), 1, 64));
    std::string_view field = std::string_view(op).substr(underscore + 1);
    if (field == "sustain") {
        env.sustain = whole(value, 0, 63);
    } else if (field == "pitch") {
        env.pitch = real(value, -12000, 12000);
    } else if (startsWith(field, "pitch_oncc")) {
        env.pitchCc.slot(modulationCc(field.substr(10))) = real(value, -12000, 12000);
    } else if (startsWith(field, "level")) {
        env.stages.slot(whole(std::string(field.substr(5)), 0, 63)).level = real(value, -1, 1);
    } else if (startsWith(field, "time")) {
        field.remove_prefix(4);
        const auto cc = field.find("_oncc");
        FlexStage& stage = env.stages.slot(whole(std::string(field.substr(0, cc)), 0, 63));
        if (cc == field.npos)
            stage.seconds = real(value, 0, 100);
        else
            stage.secondsCc.slot(modulationCc(field.substr(cc + 5))) = real(value, -100, 100);
    } else {
        return false;
    }
    return true;
}

bool ccFadeOpcode(Region& r, const std::string& op, const std::string& value)
{
    if (op == "xf_cccurve") {
        r.amp.ccFadePower = powerCurve(value);
        return true;
    }
    static constexpr std::pair<std::string_view, int Crossfade::*> kFields[] = {
        {"xfin_locc", &Crossfade::inLo}, {"xfin_hicc", &Crossfade::inHi},
        {"xfout_locc", &Crossfade::outLo}, {"xfout_hicc", &Crossfade::outHi},
    };
    for (const auto& [prefix, member] : kFields)
        if (startsWith(op, prefix)) {
            const int cc = whole(op.substr(prefix.size()), 0, 127);
            r.amp.ccFades.slot(cc).*member = whole(value, 0, 127);
            return true;
        }
    return false;
}

// var<N>_<target> opcodes of SFZ v2 variables that sfizz 1.2.3 reads and ignores.
bool ignoredVariable(const std::string& op)
{
    if (op.compare(0, 3, "var") != 0)
        return false;
    const auto first = op.find_first_not_of("0123456789", 3);
    if (first == 3 || first == op.npos || op[first] != '_')
        return false;
    const std::string_view target(op.data() + first + 1, op.size() - first - 1);
    return target == "cutoff" || target == "mod" || startsWith(target, "oncc") || startsWith(target, "curvecc") ||
        startsWith(target, "eq");
}

// ---- region opcodes by exact name ----------------------------------------------------

// What a region accumulates while its opcodes apply: the region, its sample name
// and its CC ranges (conditions and triggers) by controller.
struct Draft {
    Region region;
    std::string sample;
    Keyed<int, CcRange> conditions, triggers;
};

using Handler = void (*)(Draft&, const std::string&);

const std::unordered_map<std::string, Handler>& exactOpcodes()
{
    static const std::unordered_map<std::string, Handler> table = [] {
        std::unordered_map<std::string, Handler> t;
        const auto add = [&t](std::initializer_list<const char*> names, Handler h) {
            for (const char* name : names)
                t.emplace(name, h);
        };
        add({"sample"}, [](Draft& d, const std::string& v) { d.sample = v; });
        // Labels and the key shorthand (applied before the scope's other opcodes).
        add({"key", "group_label", "master_label", "global_label", "region_label", "sw_label"},
            [](Draft&, const std::string&) {});
        add({"lokey"}, [](Draft& d, const std::string& v) { d.region.select.keys.lo = v == "-1" ? 0 : noteNumber(v); });
        add({"hikey"}, [](Draft& d, const std::string& v) {
            d.region.select.onNotes = v != "-1";
            d.region.select.keys.hi = d.region.select.onNotes ? noteNumber(v) : 127;
        });
        add({"pitch_keycenter"}, [](Draft& d, const std::string& v) { d.region.select.center = noteNumber(v); });
        add({"lovel"}, [](Draft& d, const std::string& v) { d.region.select.velocities.lo = whole(v, 0, 127); });
        add({"hivel"}, [](Draft& d, const std::string& v) { d.region.select.velocities.hi = whole(v, 0, 127); });
        add({"lochan", "hichan"}, [](Draft&, const std::string& v) { (void)whole(v, 1, 16); });
        add({"volume"}, [](Draft& d, const std::string& v) { d.region.amp.volumeDb += real(v, -144, 60); });
        add({"amplitude"}, [](Draft& d, const std::string& v) { d.region.amp.linear *= real(v, 0, 10000) / 100; });
        add({"amp_veltrack"}, [](Draft& d, const std::string& v) { d.region.amp.velocityTrack = real(v, -100, 100) / 100; });
        add({"amp_random"}, [](Draft& d, const std::string& v) { d.region.amp.randomDb = real(v, -24, 24); });
        add({"pitch_random"}, [](Draft& d, const std::string& v) { d.region.pitch.random = real(v, -12000, 12000); });
        add({"pan"}, [](Draft& d, const std::string& v) { d.region.amp.pan = real(v, -100, 100) / 100; });
        add({"width"}, [](Draft& d, const std::string& v) { d.region.amp.width = real(v, -100, 100) / 100; });
        add({"position"}, [](Draft& d, const std::string& v) { d.region.amp.position = real(v, -100, 100) / 100; });
        add({"xfin_lokey"}, [](Draft& d, const std::string& v) { d.region.amp.keyFade.inLo = noteNumber(v); });
        add({"xfin_hikey"}, [](Draft& d, const std::string& v) { d.region.amp.keyFade.inHi = noteNumber(v); });
        add({"xfout_lokey"}, [](Draft& d, const std::string& v) { d.region.amp.keyFade.outLo = noteNumber(v); });
        add({"xfout_hikey"}, [](Draft& d, const std::string& v) { d.region.amp.keyFade.outHi = noteNumber(v); });
        add({"xfin_lovel"}, [](Draft& d, const std::string& v) { d.region.amp.velocityFade.inLo = whole(v, 0, 127); });
        add({"xfin_hivel"}, [](Draft& d, const std::string& v) { d.region.amp.velocityFade.inHi = whole(v, 0, 127); });
        add({"xfout_lovel"}, [](Draft& d, const std::string& v) { d.region.amp.velocityFade.outLo = whole(v, 0, 127); });
        add({"xfout_hivel"}, [](Draft& d, const std::string& v) { d.region.amp.velocityFade.outHi = whole(v, 0, 127); });
        add({"xf_keycurve"}, [](Draft& d, const std::string& v) { d.region.amp.keyFade.power = powerCurve(v); });
        add({"xf_velcurve"}, [](Draft& d, const std::string& v) { d.region.amp.velocityFade.power = powerCurve(v); });
        add({"tune", "pitch"}, [](Draft& d, const std::string& v) { d.region.pitch.tune = real(v, -1200, 1200); });
        add({"transpose"}, [](Draft& d, const std::string& v) { d.region.pitch.transpose = whole(v, -127, 127); });
        add({"pitch_keytrack"}, [](Draft& d, const std::string& v) { d.region.pitch.keyTrack = real(v, -1200, 1200); });
        add({"bend_up", "bendup"}, [](Draft& d, const std::string& v) { d.region.pitch.bendUp = real(v, -12000, 12000); });
        add({"bend_down", "benddown"},
            [](Draft& d, const std::string& v) { d.region.pitch.bendDown = real(v, -12000, 12000); });
        add({"bend_smooth"}, [](Draft& d, const std::string& v) { d.region.pitch.bendSmoothMs = whole(v, 0, 10000); });
        add({"delay"}, [](Draft& d, const std::string& v) { d.region.rules.delay = real(v, 0, 100); });
        add({"group"}, [](Draft& d, const std::string& v) { d.region.rules.group = whole64(v, -INT32_MAX, UINT32_MAX); });
        add({"note_polyphony"}, [](Draft& d, const std::string& v) { d.region.rules.notePolyphony = whole(v, 1, 256); });
        add({"note_selfmask"}, [](Draft& d, const std::string& v) { d.region.rules.selfMask = v == "mask" || onOff(v); });
        add({"oscillator_phase"},
            [](Draft& d, const std::string& v) { d.region.source.oscillatorPhase = real(v, -1000, 1000); });
        add({"off_by", "offby"}, [](Draft& d, const std::string& v) {
            d.region.rules.offBy = whole64(v, -INT32_MAX, UINT32_MAX);
            d.region.rules.chokedByGroup = true;
        });
        add({"off_mode", "offmode"}, [](Draft& d, const std::string& v) {
            if (v == "fast") d.region.rules.offMode = OffKind::fast;
            else if (v == "normal") d.region.rules.offMode = OffKind::normal;
            else if (v == "time") d.region.rules.offMode = OffKind::time;
            else fail("unsupported off mode " + v);
        });
        add({"off_time"}, [](Draft& d, const std::string& v) {
            d.region.rules.offTime = real(v, 0, 100);
            d.region.rules.offMode = OffKind::time;
        });
        add({"offset"}, [](Draft& d, const std::string& v) { d.region.source.offset = whole(v, 0, INT32_MAX - 1); });
        add({"offset_random"},
            [](Draft& d, const std::string& v) { d.region.source.offsetRandom = whole(v, 0, INT32_MAX - 1); });
        add({"end"}, [](Draft& d, const std::string& v) { d.region.source.end = whole(v, 0, INT32_MAX - 1); });
        add({"loop_start", "loopstart"},
            [](Draft& d, const std::string& v) { d.region.source.loopStart = whole(v, 0, INT32_MAX - 1); });
        add({"loop_end", "loopend"},
            [](Draft& d, const std::string& v) { d.region.source.loopEnd = whole(v, 0, INT32_MAX - 1); });
        add({"loop_crossfade"},
            [](Draft& d, const std::string& v) { d.region.source.loopCrossfade = std::max(.001f, real(v, 0, 100)); });
        add({"loop_type", "looptype"}, [](Draft&, const std::string& v) {
            // Direction hints have no effect in sfizz 1.2.3; only their spelling is checked.
            if (v != "forward" && v != "alternate" && v != "backward")
                fail("unknown loop direction hint " + v);
        });
        add({"ampeg_delay"}, [](Draft& d, const std::string& v) { d.region.ampEnvelope.stage[kDelay] = real(v, 0, 100); });
        add({"ampeg_attack"}, [](Draft& d, const std::string& v) { d.region.ampEnvelope.stage[kAttack] = real(v, 0, 100); });
        add({"ampeg_hold"}, [](Draft& d, const std::string& v) { d.region.ampEnvelope.stage[kHold] = real(v, 0, 100); });
        add({"ampeg_decay"}, [](Draft& d, const std::string& v) { d.region.ampEnvelope.stage[kDecay] = real(v, 0, 100); });
        add({"ampeg_sustain"},
            [](Draft& d, const std::string& v) { d.region.ampEnvelope.stage[kSustain] = real(v, 0, 100) / 100; });
        add({"ampeg_start"},
            [](Draft& d, const std::string& v) { d.region.ampEnvelope.stage[kStart] = real(v, 0, 100) / 100; });
        add({"ampeg_release"},
            [](Draft& d, const std::string& v) { d.region.ampEnvelope.stage[kRelease] = real(v, 0, 100); });
        add({"ampeg_dynamic"}, [](Draft& d, const std::string& v) { d.region.ampEnvelope.dynamic = onOff(v); });
        add({"ampeg_attack_shape", "ampeg_release_shape"}, [](Draft&, const std::string&) {});
        add({"rt_decay"}, [](Draft& d, const std::string& v) { d.region.rules.releaseDecay = real(v, 0, 200); });
        add({"rt_dead"}, [](Draft& d, const std::string& v) { d.region.rules.releaseDead = onOff(v); });
        add({"sustain_sw"}, [](Draft& d, const std::string& v) { d.region.rules.pedal = onOff(v); });
        add({"sustain_cc"}, [](Draft& d, const std::string& v) { d.region.rules.pedalCc = whole(v, 0, 127); });
        add({"sustain_lo"}, [](Draft& d, const std::string& v) { d.region.rules.pedalLow = whole(v, 0, 127); });
        add({"seq_length"}, [](Draft& d, const std::string& v) { d.region.select.sequenceLength = whole(v, 1, 1000000); });
        add({"seq_position"}, [](Draft& d, const std::string& v) {
            d.region.select.sequencePosition = whole(v, 1, 1000000);
            d.region.select.sequenceExplicit = true;
        });
        add({"sw_default"}, [](Draft& d, const std::string& v) { d.region.select.switchDefault = noteNumber(v); });
        add({"sw_down"}, [](Draft& d, const std::string& v) { d.region.select.switchDown = noteNumber(v); });
        add({"sw_up"}, [](Draft& d, const std::string& v) { d.region.select.switchUp = noteNumber(v); });
        add({"sw_previous"}, [](Draft& d, const std::string& v) { d.region.select.switchPrevious = noteNumber(v); });
        add({"sw_lokey", "sw_hikey"}, [](Draft&, const std::string& v) { (void)noteNumber(v); });
        add({"sw_last"}, [](Draft& d, const std::string& v) {
            Selection& s = d.region.select;
            if (!s.switchIsRange)
                s.switchLo = s.switchHi = noteNumber(v);
        });
        add({"sw_lolast"}, [](Draft& d, const std::string& v) {
            Selection& s = d.region.select;
            const int note = noteNumber(v);
            if (!s.switchIsRange)
                s.switchLo = s.switchHi = note;
            s.switchLo = note;
            s.switchIsRange = true;
        });
        add({"sw_hilast"}, [](Draft& d, const std::string& v) {
            Selection& s = d.region.select;
            const int note = noteNumber(v);
            if (!s.switchIsRange)
                s.switchLo = s.switchHi = note;
            s.switchHi = note;
            s.switchIsRange = true;
        });
        add({"lorand"}, [](Draft& d, const std::string& v) { d.region.select.randomLo = real(v, 0, 1); });
        add({"hirand"}, [](Draft& d, const std::string& v) { d.region.select.randomHi = real(v, 0, 1); });
        add({"trigger"}, [](Draft& d, const std::string& v) {
            static const std::map<std::string, Trigger> kTriggers{
                {"attack", Trigger::attack}, {"release", Trigger::release}, {"release_key", Trigger::releaseKey},
                {"first", Trigger::first}, {"legato", Trigger::legato}};
            d.region.select.trigger = kTriggers.at(v);
        });
        add({"loop_mode"}, [](Draft& d, const std::string& v) {
            static const std::map<std::string, LoopKind> kModes{
                {"no_loop", LoopKind::off}, {"one_shot", LoopKind::oneShot},
                {"loop_continuous", LoopKind::continuous}, {"loop_sustain", LoopKind::sustain}};
            d.region.source.loop = kModes.at(v);
        });
        return t;
    }();
    return table;
}

void applyVelocityPoint(Draft& d, const std::string& op, const std::string& v)
{
    const int velocity = whole(op.substr(13), 0, 127);
    const float value = real(v, 0, 1);
    auto& curve = d.region.amp.velocityCurve;
    const auto point = std::find_if(curve.begin(), curve.end(), [&](const auto& p) { return p.first == velocity; });
    if (point == curve.end())
        curve.emplace_back(velocity, value);
    else
        point->second = value;
}

// One opcode of a region's effective set.
void applyOpcode(Draft& d, const std::string& op, const std::string& v)
{
    const auto& table = exactOpcodes();
    if (const auto handler = table.find(op); handler != table.end()) {
        handler->second(d, v);
        return;
    }
    if (op.compare(0, 13, "amp_velcurve_") == 0) {
        applyVelocityPoint(d, op, v);
        return;
    }
    Region& r = d.region;
    if (bindable(r, op, v) || filterOpcode(r, op, v) || eqOpcode(r, op, v) || lfoOpcode(r, op, v) ||
        auxEnvelope(r, op, v) || flexOpcode(r, op, v) || ccFadeOpcode(r, op, v) || ignoredVariable(op))
        return;
    // CC ranges: locc<N>/hicc<N> condition the region, on_locc<N>/on_hicc<N> trigger it.
    const bool trigger = op.compare(0, 3, "on_") == 0;
    const size_t at = trigger ? 3 : 0;
    if (op.compare(at, 4, "locc") != 0 && op.compare(at, 4, "hicc") != 0)
        fail("unsupported SFZ opcode");
    const auto cc = static_cast<uint8_t>(whole(op.substr(at + 4), 0, 127));
    auto& ranges = trigger ? d.triggers : d.conditions;
    CcRange* range = const_cast<CcRange*>(ranges.find(cc));
    if (!range) {
        ranges.slot(cc) = CcRange{cc, 0, 127};
        range = &ranges.slot(cc);
    }
    (op[at] == 'l' ? range->lo : range->hi) = static_cast<uint8_t>(whole(v, 0, 127));
}

// ---- the lexer and the scopes -----------------------------------------------------------

class Reader {
public:
    Reader(Path root, SampleBank& bank) : root_(std::move(root)), bank_(bank) {}

    Instrument read(const Path& path)
    {
        lex(path, 0);
        closeBlock();
        if (out_.regions.empty())
            fail("no playable SFZ regions in " + path.u8string());
        return std::move(out_);
    }

private:
    Path root_, samplePath_;
    SampleBank& bank_;
    Instrument out_;
    std::string header_;
    Scope global_, master_, group_, region_, curve_;
    std::map<std::string, std::string> defines_;
    int nextCurve_ = 7;
    bool indexedCurves_ = false;

    // $NAME references replaced by their #define values.
    std::string expand(std::string text) const
    {
        for (size_t at = 0; (at = text.find('$', at)) != text.npos;) {
            size_t end = at + 1;
            while (end < text.size() && opcodeChar(text[end]))
                ++end;
            const std::string name = text.substr(at, end - at);
            const auto found = defines_.find(name);
            if (found == defines_.end())
                fail("undefined SFZ macro " + name);
            text.replace(at, end - at, found->second);
            at += found->second.size();
        }
        return text;
    }

    void lex(const Path& file, int depth)
    {
        if (depth >= 32)
            fail("too many nested SFZ includes");
        std::ifstream in(file, std::ios::binary);
        if (!in)
            fail("cannot open SFZ " + file.u8string());
        const std::string text{std::istreambuf_iterator<char>(in), {}};
        const std::string_view src(text);
        size_t at = src.substr(0, 3) == "\xef\xbb\xbf" ? 3 : 0;
        try {
            while (at < src.size()) {
                at = src.find_first_not_of(kSpaces, at);
                if (at == src.npos)
                    break;
                if (src.substr(at, 2) == "//")
                    at = src.find('\n', at);
                else if (src[at] == '<')
                    at = lexHeader(src, at);
                else if (src[at] == '#')
                    at = lexDirective(src, at, file, depth);
                else
                    at = lexOpcode(src, at);
            }
        } catch (const std::exception& error) {
            const auto line = 1 + std::count(src.begin(), src.begin() + std::min(at, src.size()), '\n');
            fail(file.u8string() + ":" + std::to_string(line) + ": " + error.what());
        }
    }

    size_t lexHeader(std::string_view src, size_t at)
    {
        const auto close = src.find('>', at + 1);
        if (close == src.npos)
            fail("unclosed SFZ header");
        openHeader(stripped(src.substr(at + 1, close - at - 1)));
        return close + 1;
    }

    size_t lexDirective(std::string_view src, size_t at, const Path& file, int depth)
    {
        const auto eol = src.find('\n', at);
        const std::string_view line = src.substr(at, eol - at);
        if (startsWith(line, "#include")) {
            const std::string target = stripped(line.substr(8));
            if (target.size() < 2 || target.front() != '"' || target.back() != '"')
                fail("expected quoted #include path");
            lex(file.parent_path() / portablePath(dequoted(expand(target))), depth + 1);
        } else if (startsWith(line, "#define")) {
            const std::string body = stripped(line.substr(7));
            const auto gap = body.find_first_of(kSpaces);
            if (body.empty() || body.front() != '$' || gap == body.npos)
                fail("invalid #define");
            defines_[body.substr(0, gap)] = expand(stripped(std::string_view(body).substr(gap)));
        } else {
            fail("unsupported SFZ directive " + std::string(line));
        }
        return eol;
    }

    // name=value: the value runs to the end of the line, a header, a comment or
    // the next name=; quotes protect spaces and those markers.
    size_t lexOpcode(std::string_view src, size_t at)
    {
        const auto nameEnd = [&](size_t from) {
            while (from < src.size() && (opcodeChar(src[from]) || src[from] == '$'))
                ++from;
            return from;
        };
        const size_t end = nameEnd(at);
        const auto equals = src.find_first_not_of(" \t", end);
        if (end == at || equals == src.npos || src[equals] != '=')
            fail("expected opcode=value");
        const std::string name = expand(std::string(src.substr(at, end - at)));
        size_t pos = equals + 1;
        bool quoted = false;
        for (; pos < src.size(); ++pos) {
            const char c = src[pos];
            if (c == '"')
                quoted = !quoted;
            if (quoted)
                continue;
            if (c == '\r' || c == '\n' || c == '<' || src.substr(pos, 2) == "//")
                break;
            if (c == ' ' || c == '\t') {
                const auto next = src.find_first_not_of(" \t", pos);
                const size_t tail = nameEnd(next);
                const auto sep = src.find_first_not_of(" \t", tail);
                if (tail != next && sep < src.size() && src[sep] == '=')
                    break;
            }
        }
        if (quoted)
            fail("unclosed quoted value for " + name);
        storeOpcode(name, dequoted(expand(stripped(src.substr(equals + 1, pos - equals - 1)))));
        return pos;
    }

    void closeBlock()
    {
        if (header_ == "curve")
            closeCurve();
        else
            closeRegion();
    }

    void openHeader(const std::string& name)
    {
        closeBlock();
        header_ = name;
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
            fail("unsupported SFZ header <" + name + ">");
        }
    }

    void setInitialCc(int cc, float value)
    {
        if (cc < 128)
            out_.startCc[size_t(cc)] = value;
        else
            out_.extendedDefaults[cc] = value;
    }

    void storeOpcode(const std::string& name, const std::string& value)
    {
        if (value.empty())
            fail("empty value for " + name);
        if (header_ == "global") global_[name] = value;
        else if (header_ == "master") master_[name] = value;
        else if (header_ == "group") group_[name] = value;
        else if (header_ == "region") region_[name] = value;
        else if (header_ == "curve") curve_[name] = value;
        else if (header_ == "control") controlOpcode(name, value);
        else fail("opcode outside SFZ header " + name);
    }

    void controlOpcode(const std::string& name, const std::string& value)
    {
        if (name == "default_path")
            samplePath_ = portablePath(value);
        else if (name.compare(0, 6, "set_cc") == 0)
            setInitialCc(whole(name.substr(6), 0, 511), real(value, 0, 127));
        else if (name.compare(0, 8, "set_hdcc") == 0)
            setInitialCc(whole(name.substr(8), 0, 511), 127 * real(value, 0, 1));
        else if (name.compare(0, 8, "label_cc") == 0)
            (void)whole(name.substr(8), 0, 511);
        else if (name.compare(0, 9, "label_key") == 0)
            (void)whole(name.substr(9), 0, 127);
        else if (name != "image" && name != "image_controls")    // display metadata
            fail("unsupported control opcode " + name);
    }

    // <curve>: v<N>=value points joined linearly over 0-127 (endpoints 0 and 1 by
    // default), stored as curve `curve_index` or the next free number from 7.
    void closeCurve()
    {
        const auto index = curve_.find("curve_index");
        if (index == curve_.end() && indexedCurves_) {
            curve_.clear();
            return;
        }
        const int id = index == curve_.end() ? nextCurve_++ : whole(index->second, 0, 255);
        indexedCurves_ |= index != curve_.end();
        std::map<int, float> knots{{0, 0.f}, {127, 1.f}};
        for (const auto& [name, value] : curve_) {
            if (name == "curve_index")
                continue;
            if (name.front() != 'v')
                fail("unsupported <curve> opcode " + name);
            knots[whole(name.substr(1), 0, 127)] = real(value, -1e16f, 1e16f);
        }
        Curve& curve = out_.curves[id];
        for (auto a = knots.begin(), b = std::next(a); b != knots.end(); ++a, ++b)
            for (int x = a->first; x <= b->first; ++x) {
                const float phase = float(x - a->first) / (b->first - a->first);
                curve[size_t(x)] = std::clamp(a->second + phase * (b->second - a->second), -1.f, 1.f);
            }
        curve_.clear();
    }

    // The effective opcodes of the closing <region>, applied scope by scope.
    Draft draftRegion() const
    {
        Draft d;
        for (const Scope* scope : {&global_, &master_, &group_, &region_}) {
            // key= sets the key range and the keycenter; the scope's specific
            // opcodes, applied after it, win.
            if (const auto key = scope->find("key"); key != scope->end()) {
                Selection& s = d.region.select;
                s.onNotes = key->second != "-1";
                s.keys.lo = s.keys.hi = s.center = s.onNotes ? noteNumber(key->second) : 60;
            }
            for (const auto& [name, value] : *scope) {
                try {
                    applyOpcode(d, name, value);
                } catch (const std::exception& error) {
                    fail(name + "=" + value + ": " + error.what());
                }
            }
        }
        return d;
    }

    void closeRegion()
    {
        if (header_ != "region")
            return;
        Draft d = draftRegion();
        const bool bare = region_.empty();
        region_.clear();
        Region& r = d.region;
        std::string& sample = d.sample;
        if (sample.empty() && bare)
            sample = "*silence";
        if (sample == "*sine") r.source.generator = CS_GEN_SINE;
        else if (sample == "*silence") r.source.generator = CS_GEN_SILENCE;
        else if (sample == "*noise") r.source.generator = CS_GEN_NOISE;
        else if (sample.empty() || sample.front() == '*') fail("missing or unsupported region sample " + sample);
        const Selection& s = r.select;
        if ((s.keys.lo > s.keys.hi && d.triggers.empty()) || s.velocities.lo > s.velocities.hi ||
            s.randomLo > s.randomHi || s.switchLo > s.switchHi)
            fail("invalid region range for " + sample);
        auto& curve = r.amp.velocityCurve;
        if (!curve.empty()) {
            std::sort(curve.begin(), curve.end());
            if (curve.front().first != 0)
                curve.insert(curve.begin(), {0, 0.f});
            if (curve.back().first != 127)
                curve.emplace_back(127, 1.f);
        }
        if (r.source.generator == CS_GEN_NONE)
            resolveSample(r, sample);
        registerRegion(d, sample);
    }

    // The sample's frames bound the region's end; an automatic loop mode takes the
    // sample's own loop (or an explicit loop_end); loop points become [start, end).
    void resolveSample(Region& r, const std::string& name)
    {
        Source& src = r.source;
        src.sampleId = bank_.describe((root_ / samplePath_ / portablePath(name)).string());
        const Sample& audio = bank_.samples[size_t(src.sampleId)];
        src.end = src.end < 0 ? audio.frames : std::min(src.end + 1, audio.frames);
        if (src.offset >= src.end)
            fail("offset past end of sample " + name);
        if (src.loop == LoopKind::unset)
            src.loop = audio.loopEnd > 0 || src.loopEnd >= 0 ? LoopKind::continuous : LoopKind::off;
        if (src.loop == LoopKind::continuous || src.loop == LoopKind::sustain) {
            if (src.loopStart < 0)
                src.loopStart = audio.loopFirst;
            src.loopEnd = src.loopEnd < 0 ? (audio.loopEnd > 0 ? audio.loopEnd : src.end)
                                          : std::min(src.loopEnd + 1, src.end);
            if (src.loopStart >= src.loopEnd || src.loopEnd > src.end || src.offset >= src.loopEnd)
                fail("invalid forward loop in " + name);
        }
    }

    void markCc(int cc)
    {
        if (cc < 128)
            out_.ccInUse[size_t(cc)] = true;
    }

    // Controllers the region listens to, checks of its modulators, and its place
    // in the key and controller indexes.
    void registerRegion(Draft& d, const std::string& name)
    {
        Region& r = d.region;
        for (const auto& [cc, range] : d.conditions) {
            if (range.lo > range.hi)
                fail("invalid CC range for " + name);
            r.select.ccConditions.push_back(range);
            markCc(cc);
        }
        for (auto& [cc, fade] : r.amp.ccFades) {
            fade.power = r.amp.ccFadePower;
            markCc(cc);
        }
        for (const CcBinding& b : r.bindings)
            markCc(b.cc);
        for (const auto& [index, lfo] : r.lfos) {
            for (const auto& [target, depth] : lfo.depth)
                enableFor(r, target);
            for (const CcBinding& b : lfo.ccs) {
                markCc(b.cc);
                enableFor(r, b.target);
            }
        }
        for (const auto& [index, env] : r.flex) {
            if (env.stages.empty() || env.stages.items.back().second.level != 0 ||
                (env.sustain >= 0 && env.sustain != env.stages.items.back().first))
                fail("flexible pitch envelope must end at a zero-level sustain point");
            for (const auto& [cc, depth] : env.pitchCc)
                markCc(cc);
            for (const auto& [stage, point] : env.stages)
                for (const auto& [cc, seconds] : point.secondsCc)
                    markCc(cc);
        }
        if (r.rules.pedal)
            markCc(r.rules.pedalCc);
        const int index = int(out_.regions.size());
        if (r.select.onNotes)
            for (int note = r.select.keys.lo; note <= r.select.keys.hi; ++note)
                out_.regionsByKey[size_t(note)].push_back(index);
        for (const auto& [cc, range] : d.triggers) {
            if (range.lo > range.hi)
                fail("invalid CC trigger range for " + name);
            r.select.ccTriggers.push_back(range);
            out_.regionsByCc[size_t(cc)].push_back(index);
            markCc(cc);
        }
        if (r.select.switchLo >= 0)
            for (int note = r.select.switchLo; note <= r.select.switchHi; ++note)
                out_.switchKey[size_t(note)] = true;
        if (r.select.switchDefault >= 0)
            out_.startSwitch = r.select.switchDefault;
        out_.anyChoke |= r.rules.chokedByGroup;
        out_.regions.push_back(std::move(r));
    }
};

} // namespace

Instrument readInstrument(const std::string& path, SampleBank& bank)
{
    const Path file = std::filesystem::u8path(path);
    return Reader(file.parent_path(), bank).read(file);
}

// A controller value (0-127, fractional between steps) through curve `curve`: a
// <curve> of the instrument, else one of the format's built-in curves 0-6.
float applyCurve(const Instrument& instrument, int curve, float value)
{
    value = std::clamp(value, 0.f, 127.f);
    const int lo = static_cast<int>(value);
    const int hi = std::min(127, lo + 1);
    const float fraction = value - lo;
    if (const auto custom = instrument.curves.find(curve); custom != instrument.curves.end())
        return custom->second[size_t(lo)] + fraction * (custom->second[size_t(hi)] - custom->second[size_t(lo)]);
    const auto builtIn = [curve](int step) {
        const float x = step / 127.f;
        switch (curve) {
        case 1: return 2 * x - 1;       // bipolar
        case 2: return 1 - x;           // inverted
        case 3: return 1 - 2 * x;       // inverted bipolar
        case 4: return x * x;
        case 5: return std::sqrt(x);
        case 6: return std::sqrt(1 - x);
        default: return x;              // linear
        }
    };
    const float a = builtIn(lo);
    return a + fraction * (builtIn(hi) - a);
}

} // namespace clayhost
