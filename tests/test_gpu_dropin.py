"""The drop-in integration end to end: GAMERA-OP's own program (src/main.c,
config.yaml, problem hooks, geometry, HDF5 output) with its step driver
replaced by gamera-op_b200/host/gop_solve.c and its ghost-fill library by the
recording gop_bc_record.c, against the unmodified reference binary on the
same input.  Both binaries are built from the reference sources by
``make -C oracle reference dropin``; the test is skipped where they were not.
"""
import numpy as np
import pytest

from conftest import NG, rel_l1

pytestmark = pytest.mark.gpu

ref_run = pytest.importorskip("ref_run")


def _need(*names):
    for nm in names:
        if not (ref_run.REF_DIR / nm).exists():
            pytest.skip(f"oracle/_ref/{nm} not built")


def _compare_dumps(a, b, n, tol):
    act = tuple(slice(NG, NG + m) for m in n)
    for slot in range(6):
        if slot == 5:
            continue  # p_S stays 0 in both
        e = rel_l1(a["gas"][0][slot][act], b["gas"][0][slot][act])
        assert e <= tol, f"gas slot {slot}: {e}"
    for slot in range(3):
        s = list(act)
        s[slot] = slice(NG, NG + n[slot] + 1)
        e = rel_l1(a["gem"][slot][tuple(s)], b["gem"][slot][tuple(s)])
        assert e <= tol, f"gem slot {slot}: {e}"


@pytest.mark.parametrize("case", [
    dict(n=(48, 48, 4), steps=60, problem="ot", coord="cart", bc="pppppp",
         env={"GOP_DOMAIN": "0,1,0,1,0,0.015625"}),
    dict(n=(20, 16, 12), steps=25, problem="blast", coord="cart", bc="ssrrfe",
         env={"GOP_CENTER": "0.1,-0.05,0.0", "GOP_B": "0.3,0.5,0.2"}),
    dict(n=(20, 16, 12), steps=25, problem="loop_sph", coord="sph", bc="eeeeee",
         env={"GOP_LOOP": "1.5,0,0.3,1e-3"}),
    # background fields B0: the reference's uniform and dipole hooks
    dict(n=(16, 16, 12), steps=20, problem="blast", coord="cart", bc="pppppp",
         env={"GOP_B0": "uniform"}),
    dict(n=(16, 16, 12), steps=20, problem="blast", coord="cart", bc="eeeeee",
         env={"GOP_B0": "dipole", "GOP_DOMAIN": "1.0,2.0,-0.5,0.5,-0.5,0.5",
              "GOP_CENTER": "1.5,0.0,0.0", "GOP_B": "0,0,0"}),
    dict(n=(20, 16, 12), steps=20, problem="loop_sph", coord="sph", bc="eeeeee",
         env={"GOP_B0": "dipole", "GOP_LOOP": "1.5,0,0.3,1e-3"}),
], ids=["ot", "blast_mixed_bc", "loop_sph", "blast_b0_uniform", "blast_b0_dipole",
        "loop_sph_b0_dipole"])
def test_dropin_solve_matches_reference_program(case):
    c = case["coord"]
    _need(f"ref_{c}_strict", f"ref_{c}_gpu")
    env = {"GOP_BC": case["bc"], **case["env"]}
    kw = dict(problem=case["problem"], coord=c, env=env, timeout=600)
    ref = ref_run.run(case["n"], case["steps"], **kw)
    gpu = ref_run.run(case["n"], case["steps"], exe=ref_run.REF_DIR / f"ref_{c}_gpu", **kw)
    assert gpu.files == ref.files  # same per-step file names
    # the step-0 dump comes from the GPU path's ghost fill (bitwise: copies)
    # and its cell-centred field (round-off: precomputed interpolation weights)
    a0, b0 = gpu.dumps[0], ref.dumps[0]
    assert np.array_equal(a0["gas"][0][:5], b0["gas"][0][:5])
    assert np.array_equal(a0["gem"][:3], b0["gem"][:3])
    scale = max(np.abs(b0["gem"][3:6]).max(), 1e-300)
    assert np.abs(a0["gem"][3:6] - b0["gem"][3:6]).max() <= 1e-13 * scale
    _compare_dumps(gpu.dumps[-1], ref.dumps[-1], case["n"], 1e-10)
    assert abs(gpu.state(-1)["time"] - ref.state(-1)["time"]) <= 1e-12 * ref.state(-1)["time"]


def test_dropin_writes_outputs_at_the_reference_times():
    _need("ref_cart_strict", "ref_cart_gpu")
    kw = dict(problem="blast", coord="cart", env={"GOP_BC": "pppppp"}, timeout=600,
              output_interval=0.01)
    ref = ref_run.run((16, 16, 16), 20, **kw)
    gpu = ref_run.run((16, 16, 16), 20, exe=ref_run.REF_DIR / "ref_cart_gpu", **kw)
    assert len(ref.files) >= 3
    assert gpu.files == ref.files
    for a, b in zip(gpu.dumps, ref.dumps):
        assert abs(float(a["time_sim"][0]) - float(b["time_sim"][0])) <= 1e-12
        _compare_dumps(a, b, (16, 16, 16), 1e-10)


def test_dropin_stops_and_logs_at_the_reference_steps():
    """The drop-in steps on the device up to the next host event (dump time,
    log time, time_stop) instead of returning to the host every step; the
    reference's status lines (step number and time) and its stop come out at
    the same steps."""
    import re
    _need("ref_cart_strict", "ref_cart_gpu")
    kw = dict(problem="blast", coord="cart", env={"GOP_BC": "pppppp"}, timeout=600,
              output_interval=0.05, time_stop=0.06)
    ref = ref_run.run((16, 16, 16), 1000, **kw)
    gpu = ref_run.run((16, 16, 16), 1000, exe=ref_run.REF_DIR / "ref_cart_gpu", **kw)
    pat = re.compile(r"Status at step (\d+): rank \d+, Time ([\d.]+)")
    a, b = pat.findall(gpu.log), pat.findall(ref.log)
    steps = [int(s) for s, _ in b]
    assert len(b) >= 3 and max(y - x for x, y in zip(steps, steps[1:])) > 1
    assert [s for s, _ in a] == [s for s, _ in b]
    for (_, ta), (_, tb) in zip(a, b):
        assert abs(float(ta) - float(tb)) <= 1e-12
    assert gpu.files == ref.files
    assert abs(gpu.state(-1)["time"] - ref.state(-1)["time"]) <= 1e-12
    assert ref.state(-1)["time"] > 0.06 and len(ref.files) == 3
