"""The oracle's plain-C restatement of the render path, pinned against the
reference's own code built for the host (oracle/_ref) and against the golden
vectors the reference's tests assert."""
import numpy as np
import pytest

from claysampler_b200 import workload


def ref_or_skip():
    from oracle import reference
    if not (reference.available() or reference.build()):
        pytest.skip("oracle/_ref (the reference built for the host) is not available")
    return reference


def test_sinc_table_matches_reference():
    from oracle import oracle
    reference = ref_or_skip()
    mine = np.zeros(48 * 2049, np.float32)
    oracle.lib().oracle_sinc_table(mine.ctypes.data)
    assert np.array_equal(mine.view(np.uint32), reference.sinc_table().reshape(-1).view(np.uint32))


def test_sinc_table_is_symmetric():
    """sinc[tap][phase] == sinc[47 - tap][2048 - phase] bit for bit: the shared-source
    kernel keeps only phases 0-1024 in shared memory and reads a phase above 1024
    as row 2048 - phase backwards."""
    from oracle import oracle
    table = np.zeros(48 * 2049, np.float32)
    oracle.lib().oracle_sinc_table(table.ctypes.data)
    table = table.reshape(48, 2049)
    mirrored = table[::-1, ::-1]
    assert np.array_equal(table.view(np.uint32), mirrored.view(np.uint32))


@pytest.mark.parametrize("tail", ["natural", "orig"])
@pytest.mark.parametrize("fixture", ["plain_small", "batch_mini"])
def test_restated_render_matches_reference_bit_for_bit(request, ref_session, fixture, tail):
    from oracle import oracle
    reference = ref_or_skip()
    jobs = request.getfixturevalue(fixture)
    plans = [ref_session.plan(j.sfz, j.midi, tail=tail) for j in jobs]
    bank = ref_session.bank()
    natural = tail == "natural"
    theirs = reference.synthesize(plans, bank, natural)
    mine = oracle.synthesize(plans, bank, natural)
    assert np.array_equal(mine.view(np.uint32 if natural else np.uint16), theirs.view(np.uint32 if natural else np.uint16))


# The FP32 resampler (48 FMAs over the FP32-rounded table, render.cu:30-61)
# against the oracle's FP64 evaluation on the unrounded table
# (renderer.cpp:365-373): its rounding error, measured on the uneven batch's
# transposed mono voices, is about 1e-7 FS (a few ULPs at the mix's peak).
FP64_RESAMPLER_BOUND = 2.5e-7


def test_fp64_resampler_bounds_the_fp32_render(tmp_path, ref_session):
    """The reference's FP32 render (restated bit for bit) of the first 16 jobs of
    the uneven batch, 87 % of whose voices run the 48-tap sinc, against the same
    render with the resampler in FP64: the difference is the FP32 resampler's
    rounding error and stays below FP64_RESAMPLER_BOUND."""
    from oracle import oracle
    jobs = workload.write_uneven_batch(tmp_path, seed=2, jobs=1024)[:16]
    plans = [ref_session.plan(j.sfz, j.midi) for j in jobs]
    bank = ref_session.bank()
    fp32 = oracle.synthesize(plans, bank)
    fp64 = oracle.synthesize(plans, bank, fp64_resampler=True)
    err = np.abs(fp32.astype(np.float64) - fp64.astype(np.float64))
    assert 0 < err.max() <= FP64_RESAMPLER_BOUND, err.max()
    assert np.sqrt(np.mean(err ** 2)) < 1e-8


def test_restated_render_pitch_and_bends(tmp_path, ref_session):
    """Variable pitch (LFO to pitch), bends, CC-driven cutoff: the reference's
    check_segments.py voice and check_tail.py's processed preset."""
    import struct
    import wave
    from oracle import oracle
    reference = ref_or_skip()
    rate = 44100
    with wave.open(str(tmp_path / "sample.wav"), "wb") as stream:
        stream.setparams((1, 2, rate, 0, "NONE", "not compressed"))
        stream.writeframes(b"".join(struct.pack("<h", round(3000 * np.sin(i * .04))) for i in range(rate)))
    sfz = tmp_path / "voice.sfz"
    sfz.write_text("<region> sample=sample.wav key=60 loop_mode=loop_continuous loop_start=0 loop_end=44099 "
                   "amp_veltrack=0 ampeg_release=1.7 cutoff=1800 resonance=3 cutoff_oncc1=3000 pitch_oncc1=37 "
                   "lfo1_freq=3 lfo1_pitch=120\n", encoding="ascii")
    data = bytes.fromhex("00 b0 40 7f 00 90 3c 64 87 40 b0 01 40 87 40 e0 00 50 87 40 80 3c 00 87 40 b0 40 00 00 ff 2f 00")
    midi = tmp_path / "long.mid"
    midi.write_bytes(b"MThd" + struct.pack(">IHHH", 6, 0, 1, 480) + b"MTrk" + struct.pack(">I", len(data)) + data)
    plans = [ref_session.plan(sfz, midi, tail="orig")]
    assert plans[0].spans["variablePitch"].any()
    bank = ref_session.bank()
    for natural in (True, False):
        theirs = reference.synthesize(plans, bank, natural)
        mine = oracle.synthesize(plans, bank, natural)
        assert np.array_equal(mine.view(np.uint32 if natural else np.uint16), theirs.view(np.uint32 if natural else np.uint16))


def test_loop_remainder_identity_is_exact():
    """The device's loop wrap computes fmod(x, period) as the remainder of x's whole
    part plus x's fraction (voice_math.cuh, loopRemainder).  Both parts are exact in
    IEEE double and their sum is the exact remainder, so the result equals fmod's
    bit for bit; checked here on the positions a loop wrap sees (whole and
    fractional, near period multiples, up to 2^32)."""
    rng = np.random.default_rng(7)
    periods = np.concatenate([rng.integers(1, 1 << 20, 4000), [1, 2, 3, 1023, 65536, (1 << 31) - 1]])
    whole = rng.integers(0, 1 << 32, periods.size).astype(np.float64)
    frac = rng.random(periods.size)
    for x in (whole, whole + frac, np.minimum(whole + 0.999999999, 4294967295.0),
              periods * rng.integers(1, 50, periods.size) + frac,
              periods * rng.integers(1, 50, periods.size) - 2.0 ** -20):
        x = x[(x >= 0) & (x < 2.0 ** 32)]
        p = periods[: x.size]
        floor = np.floor(x)
        restated = (floor.astype(np.uint64) % p.astype(np.uint64)).astype(np.float64) + (x - floor)
        assert np.array_equal(restated.view(np.uint64), np.fmod(x, p.astype(np.float64)).view(np.uint64))
