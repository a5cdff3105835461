"""GPU parity of the B200 DDTR path, called through the C ABI.

For every seeded case of tests/golden/cases.py the pipeline runs through the
reference-facing entry points (aa_py_pipeline_api, bind, run loop,
aa_py_buffer) and its float DM-time output is compared
  * with the CPU oracle: bit-exact when nchans*bin is a power of two (the
    reference's fast-math division is exact there); otherwise the integer
    channel sums must agree exactly (where they stay below 2^24; larger fp32
    sums of 16-bit data are rounded) and the float within 2 ulp (the oracle
    divides with IEEE division, the device with the reference's fast-math
    division);
  * with the reference's own GPU output (golden SHA-256 per DM range,
    tests/golden/ddtr_golden.json): bit-exact.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import cases as C

pytestmark = pytest.mark.gpu

LIGHT = [n for n, c in C.CASES.items() if not c.get("heavy")]


def run_pipeline(aa, case, x, stride_mode=0, variant=0, explicit_setup=False, **opts):
    md = aa.filterbank_metadata_struct(0.0, case["tsamp"], case["fch1"], case["foff"], case["nbits"],
                                       case["nsamp"], case["nchans"], 0.0)
    comps = aa.aa_py_pipeline_components(True, False, False, False)
    o = aa.aa_py_pipeline_component_options()
    o.copy_ddtr_data_to_host = True
    pipe = aa.aa_py_pipeline(comps, o, md, np.ascontiguousarray(x.reshape(-1)), 0)
    pipe.set_options(stride_mode=stride_mode, free_memory=C.strategy_free_memory(case), **opts)
    pipe.set_kernel_variant(variant)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in case["plan"]])
    assert pipe.bind_ddtr_plan(plan), pipe.last_error()
    if explicit_setup:
        assert pipe.setup() and pipe.setup(), pipe.last_error()
    steps = 0
    while pipe.run():
        steps += 1
        assert pipe.status_code() != aa.STATUS_ERROR, pipe.last_error()
    assert pipe.status_code() == aa.STATUS_FINISHED, pipe.last_error()
    outs = [a.copy() for a in pipe.output_arrays()]
    info = [pipe.range_info(r) for r in range(len(case["plan"]))]
    launches = pipe.kernel_launches()
    pipe.cleanUp()
    pipe.delete()
    plan.delete()
    return outs, info, steps, launches


def oracle_run(oracle_mod, case, x, stride_mode=0):
    s = oracle_mod.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                            case["nbits"], C.strategy_free_memory(case))
    outs, kern = oracle_mod.run_ddtr(x, s, case["nchans"], case["nsamp"], case["tsamp"], case["nbits"],
                                     stride_mode=stride_mode)
    return s, outs, kern


def assert_matches_oracle(case, s, got, want, kern):
    for r in range(len(want)):
        g, w = got[r], want[r]
        assert g.shape == w.shape, (r, g.shape, w.shape)
        inbin = s.dm[r][3]
        div = case["nchans"] * (1 if kern[r][0] == 2 else inbin)
        if div & (div - 1) == 0:
            bad = np.flatnonzero(g.view(np.uint32) != w.view(np.uint32))
            assert bad.size == 0, f"range {r}: {bad.size} outputs differ, first at {np.unravel_index(bad[0], g.shape)}"
        else:
            sg = np.rint(g.astype(np.float64) * div)
            sw = np.rint(w.astype(np.float64) * div)
            if np.abs(sw).max() < 2**24:  # fp32 sums above 2^24 are rounded, not integers
                assert np.array_equal(sg, sw), f"range {r}: integer sums differ"
            ulp = np.abs(g.view(np.int32).astype(np.int64) - w.view(np.int32).astype(np.int64))
            assert ulp.max() <= 2, f"range {r}: {ulp.max()} ulp"


@pytest.mark.parametrize("variant", [1, 2, 0])
@pytest.mark.parametrize("name", LIGHT)
def test_pipeline_matches_oracle(aa, oracle_mod, cuda_device, name, variant):
    case = C.CASES[name]
    x = C.make_input(case)
    s, want, kern = oracle_run(oracle_mod, case, x)
    got, info, steps, launches = run_pipeline(aa, case, x, variant=variant)
    assert steps == s.num_tchunks * len(case["plan"]) + 1
    assert launches > 0
    for r in range(len(case["plan"])):
        assert info[r]["kind"] == oracle_mod.KERNEL_NAMES[kern[r][0]]
    assert_matches_oracle(case, s, got, want, kern)


@pytest.mark.parametrize("variant", [1, 2, 0])
@pytest.mark.parametrize("name", list(C.CASES))
def test_pipeline_matches_reference_gpu(aa, golden_ddtr, cuda_device, name, variant):
    if name not in golden_ddtr:
        pytest.skip("case not in the golden file")
    case = C.CASES[name]
    rec = golden_ddtr[name]
    x = C.make_input(case)
    got, _, _, _ = run_pipeline(aa, case, x, variant=variant)
    for r, rr in enumerate(rec["ranges"]):
        g = got[r]
        assert list(g.shape) == rr["shape"]
        if hashlib.sha256(g.tobytes()).hexdigest() != rr["sha256"]:
            bad = [(i, j) for i, j, bits in rr["samples"] if int(g[i, j].view(np.uint32)) != bits]
            pytest.fail(f"range {r}: output differs from the reference GPU ({len(bad)}/{len(rr['samples'])} "
                        f"sampled values differ, e.g. {bad[:3]})")


@pytest.mark.parametrize("name", ["shared8_binned", "shared8_2bit", "shared16"])
def test_true_stride_mode_matches_oracle(aa, oracle_mod, cuda_device, name):
    """The corrected binning (true row stride, repeated x2 steps)."""
    case = C.CASES[name]
    x = C.make_input(case)
    s, want, kern = oracle_run(oracle_mod, case, x, stride_mode=1)
    got, _, _, _ = run_pipeline(aa, case, x, stride_mode=1)
    assert_matches_oracle(case, s, got, want, kern)


@pytest.mark.parametrize("tile_words,group_dms,variant", [(2, 64, 1), (4, 32, 1), (4, 16, 1), (2, 8, 1), (2, 64, 2),
                                                           (4, 64, 2)])
def test_tile_shapes_agree(aa, oracle_mod, cuda_device, tile_words, group_dms, variant):
    case = C.CASES["shared8_binned"]
    x = C.make_input(case)
    s, want, kern = oracle_run(oracle_mod, case, x)
    got, info, _, _ = run_pipeline(aa, case, x, variant=variant, tile_words=tile_words, group_dms=group_dms)
    assert info[0]["group_dms"] == group_dms
    assert info[0]["kernel"] == ("quad" if variant == 2 else "phase")
    assert_matches_oracle(case, s, got, want, kern)


@pytest.mark.parametrize("name,variant,kernel", [("shared8_binned", 0, "quad|quadsp"), ("shared8_binned", 1, "phase"),
                                                 ("shared8_binned", 2, "quad"),
                                                 ("shared8_nch3000", 0, "sub|quad|quadsp"),
                                                 ("shared8_nch3000", 4, "quadws"), ("shared8_nch3000", 5, "quadsp"),
                                                 ("shared8_binned", 6, "quad"), ("shared8_binned", 7, "quad"),
                                                 ("shared8_nch3000", 6, "quad"), ("shared8_nch3000", 7, "quad"),
                                                 ("shared8_nch3000", 8, "quad"), ("shared8_binned", 8, "quad"),
                                                 ("shared8_nch3000", 9, "quad"), ("shared8_binned", 9, "quad"),
                                                 ("shared8_nch3000", 10, "quad"), ("shared8_binned", 10, "quad"),
                                                 ("shared8_nch3000", 11, "quad"), ("shared8_binned", 11, "quad"),
                                                 ("shared8_nch3000", 12, "quad"), ("shared8_binned", 12, "quad"),
                                                 ("shared8_nch3000", 3, "sub"), ("shared8_nch3000", 2, "quad"),
                                                 ("shared16", 0, "f32"), ("shared16", 1, "gather"),
                                                 ("cache16", 2, "f32")])
def test_kernel_choice(aa, oracle_mod, cuda_device, name, variant, kernel):
    """Which kernel a range runs under each variant setting (with both staged
    one-byte kernels available the autotuner times them and keeps the faster);
    results agree."""
    case = C.CASES[name]
    x = C.make_input(case)
    s, want, kern = oracle_run(oracle_mod, case, x)
    got, info, _, _ = run_pipeline(aa, case, x, variant=variant)
    assert all(i["kernel"] in kernel.split("|") for i in info), [i["kernel"] for i in info]
    assert_matches_oracle(case, s, got, want, kern)


@pytest.mark.parametrize("name", [n for n in LIGHT if C.CASES[n]["nbits"] <= 8])
def test_autotuned_tile_shape_matches_oracle(aa, oracle_mod, cuda_device, name):
    """With the autotuner on, every channel-quad range runs the tile shape and
    flavour it timed fastest (a 64 x 512 or 64 x 256 output tile; flavours
    6 and 7 only where no entry is on the per-byte path); results agree."""
    case = C.CASES[name]
    x = C.make_input(case)
    s, want, kern = oracle_run(oracle_mod, case, x)
    got, info, _, _ = run_pipeline(aa, case, x, variant=0)
    for i in info:
        if i["kernel"] == "quad":
            assert i["tile"] in ([64, 512], [64, 256]), i
            assert i["flavour"] in (0, 1, 2, 4, 6, 7), i
            assert i["dms_per_warp"] == (8 if i["tile"][1] == 256 and i["flavour"] == 0 else 4), i
        else:
            assert i["flavour"] == -1, i
    assert_matches_oracle(case, s, got, want, kern)


@pytest.mark.parametrize("name", ["shared8_binned", "shared16"])
def test_tuned_choices_kept_for_the_next_pipeline(aa, oracle_mod, cuda_device, tmp_path, name):
    """The autotuner's choices are kept per range shape: after a round trip
    through a file, a second pipeline of the same shape (set up explicitly,
    twice: set-up is idempotent) takes them without timing, adds no entry,
    runs the same kernel shapes and gives the same bits as the first and as
    the oracle; choices that do not fit the range are not taken."""
    case = C.CASES[name]
    x = C.make_input(case)
    aa.tuned_ranges(clear=True)
    first, info1, _, _ = run_pipeline(aa, case, x, variant=0)
    kept = aa.tuned_ranges()
    assert kept >= 1
    # through a file, as another process would take them
    path = str(tmp_path / "tuned.txt")
    assert aa.save_tuned_ranges(path) == kept
    aa.tuned_ranges(clear=True)
    assert aa.load_tuned_ranges(path) == kept
    used = aa.tuned_ranges_used()
    second, info2, _, _ = run_pipeline(aa, case, x, variant=0, explicit_setup=True)
    assert aa.tuned_ranges() == kept
    assert aa.tuned_ranges_used() - used >= kept
    assert info2 == info1
    for a, b in zip(first, second):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    s, want, kern = oracle_run(oracle_mod, case, x)
    assert_matches_oracle(case, s, second, want, kern)
    # an edited file (an unknown kernel in every entry): its choices are not
    # taken, the ranges are timed again, the output is the same
    lines = open(path).read().splitlines()
    fields = [ln.split() for ln in lines[1:]]
    with open(path, "w") as f:
        f.write("\n".join([lines[0]] + [" ".join(v[:-10] + ["9"] + v[-9:]) for v in fields]) + "\n")
    aa.tuned_ranges(clear=True)
    assert aa.load_tuned_ranges(path) == kept
    used = aa.tuned_ranges_used()
    third, _, _, _ = run_pipeline(aa, case, x, variant=0)
    assert aa.tuned_ranges_used() == used
    for a, b in zip(first, third):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


WS_CASES = [n for n in LIGHT if C.CASES[n]["nbits"] <= 8]
WS_REFUSED = "warp-specialised channel-quad kernel cannot run"


@pytest.mark.parametrize("name", WS_CASES)
def test_warp_specialised_quad_matches_oracle(aa, oracle_mod, golden_ddtr, cuda_device, name):
    """Variant 4 forces the warp-specialised channel-quad kernel (k_ddtr_quadws)
    on one-byte data: bit-identical to the oracle and to the reference GPU
    output.  Ranges with (quad, DM) entries on the per-byte path are refused."""
    case = C.CASES[name]
    x = C.make_input(case)
    try:
        got, info, _, _ = run_pipeline(aa, case, x, variant=4)
    except AssertionError as e:
        assert WS_REFUSED in str(e), str(e)
        pytest.skip(f"refused: {e}")
    assert all(i["kernel"] == "quadws" for i in info), [i["kernel"] for i in info]
    s, want, kern = oracle_run(oracle_mod, case, x)
    assert_matches_oracle(case, s, got, want, kern)
    for r, rr in enumerate(golden_ddtr.get(name, {}).get("ranges", [])):
        assert hashlib.sha256(got[r].tobytes()).hexdigest() == rr["sha256"], f"range {r} differs from the reference GPU"


def test_warp_specialised_quad_runs_the_plain_cases(aa, cuda_device):
    """Without two-level class delays in a group every entry has a pre-skewed
    row: the warp-specialised kernel takes these cases."""
    ran = []
    for name in ("cache8", "shared8_nch3000", "fma_probe"):
        case = C.CASES[name]
        try:
            _, info, _, _ = run_pipeline(aa, case, C.make_input(case), variant=4)
            ran.append(name)
        except AssertionError as e:
            assert WS_REFUSED in str(e), str(e)
    assert ran, "the warp-specialised kernel ran none of the cases"


SP_REFUSED = "split-phase channel-quad kernel cannot run"


@pytest.mark.parametrize("name", WS_CASES)
def test_split_phase_quad_matches_oracle(aa, oracle_mod, golden_ddtr, cuda_device, name):
    """Variant 5 forces the split-phase channel-quad kernel (k_ddtr_quadsp) on
    one-byte data: bit-identical to the oracle and to the reference GPU
    output.  Ranges with (quad, DM) entries on the per-byte path are refused."""
    case = C.CASES[name]
    x = C.make_input(case)
    try:
        got, info, _, _ = run_pipeline(aa, case, x, variant=5)
    except AssertionError as e:
        assert SP_REFUSED in str(e), str(e)
        pytest.skip(f"refused: {e}")
    assert all(i["kernel"] == "quadsp" for i in info), [i["kernel"] for i in info]
    s, want, kern = oracle_run(oracle_mod, case, x)
    assert_matches_oracle(case, s, got, want, kern)
    for r, rr in enumerate(golden_ddtr.get(name, {}).get("ranges", [])):
        assert hashlib.sha256(got[r].tobytes()).hexdigest() == rr["sha256"], f"range {r} differs from the reference GPU"


@pytest.mark.parametrize("name", WS_CASES)
def test_quad_pair_rows_match_oracle(aa, oracle_mod, golden_ddtr, cuda_device, name):
    """Variant 8 runs the channel-quad pair body (rows summed over the quad,
    16-bit pairs) on every range without per-byte entries and the channel-quad
    kernel on the others: bit-identical to the oracle and to the reference GPU."""
    case = C.CASES[name]
    x = C.make_input(case)
    got, info, _, _ = run_pipeline(aa, case, x, variant=8)
    assert all(i["kernel"] == "quad" for i in info), [i["kernel"] for i in info]
    s, want, kern = oracle_run(oracle_mod, case, x)
    assert_matches_oracle(case, s, got, want, kern)
    for r, rr in enumerate(golden_ddtr.get(name, {}).get("ranges", [])):
        assert hashlib.sha256(got[r].tobytes()).hexdigest() == rr["sha256"], f"range {r} differs from the reference GPU"


def test_split_phase_quad_runs_the_plain_cases(aa, cuda_device):
    """The split-phase kernel takes the cases whose every entry has a
    pre-skewed row."""
    ran = []
    for name in ("cache8", "shared8_nch3000", "fma_probe"):
        case = C.CASES[name]
        try:
            _, info, _, _ = run_pipeline(aa, case, C.make_input(case), variant=5)
            ran.append(name)
        except AssertionError as e:
            assert SP_REFUSED in str(e), str(e)
    assert ran, "the split-phase kernel ran none of the cases"


def test_subband_kernel_refused_where_patterns_do_not_fit(aa, cuda_device):
    """512 channels of 0.59 MHz give up to 33 skew patterns per 16-channel
    subband and 64-DM group: more than the subband kernel holds."""
    case = C.CASES["shared8_binned"]
    x = C.make_input(case)
    with pytest.raises(AssertionError, match="subband kernel cannot run range 0"):
        run_pipeline(aa, case, x, variant=3)


def test_kat_fake_signal(aa, oracle_mod, cuda_device):
    """tests/test_ddtr_fakesignal_single.cpp:109-117 with fixed seeds: all 128
    channels of the injected pulse align, so the output is exactly 255."""
    rng = np.random.Generator(np.random.PCG64(77))
    case = dict(nchans=128, nbits=8, fch1=1550.0, foff=-300.0 / 128, tsamp=6.4e-5, nsamp=int(2 / 6.4e-5),
                plan=[(0, 250.0, 1, 1, 1)], free_memory=0)
    s = oracle_mod.strategy(case["plan"], 128, case["nsamp"], 1550.0, case["foff"], 6.4e-5, 8, 180 * 2**30)
    hits = 0
    for _ in range(5):
        dm_position = float(int(rng.integers(0, 200)))
        start = int(rng.integers(0, 10)) * 1000 + int(rng.integers(0, 10)) * 100 + int(rng.integers(0, 10)) * 10
        x, _ = oracle_mod.fake_signal(128, case["nsamp"], 6.4e-5, s.dmshifts, s.maxshift, dm_position,
                                      int(1 / (6.4e-5 * 25)), start, 0.5)
        x = x.reshape(case["nsamp"], 128)
        got, _, _, _ = run_pipeline(aa, case, x)
        want, _ = oracle_mod.run_ddtr(x, s, 128, case["nsamp"], 6.4e-5, 8)
        assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32))
        hits += int(got[0][int(dm_position) // 1, start] == 255.0)
    assert hits == 5
