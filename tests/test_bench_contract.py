"""bench.py on the CPU: the compulsory-byte model behind its roofline
fields, and the JSON line of the reference arm (GAMERA-OP's own Release
build timed on the host cores; needs oracle/_ref built from the reference
sources)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def test_compulsory_bytes_per_launch():
    import bench
    n = (64, 48, 32)
    cells = 64 * 48 * 32
    faces = cells + 48 * 32  # one launch's faces along i
    ext = 73 * 57 * 41
    for mixed, w in ((False, 8), (True, 4)):
        # entropy channel off (every measured problem): 5 gas fields, 8 fluxes
        assert bench.algorithmic_bytes("flux", n, mixed) == 27 * w * faces
        assert bench.algorithmic_bytes("update", n, mixed) == (16 * 8 + 27 * w) * cells
        assert bench.algorithmic_bytes("ab2", n, mixed) == (16 * 8 + (14 + (8 if mixed else 0)) * w) * ext
        # with it: 6 gas fields, 9 fluxes
        assert bench.algorithmic_bytes("flux", n, mixed, ps_live=True) == 30 * w * faces
        assert bench.algorithmic_bytes("update", n, mixed, ps_live=True) == (18 * 8 + 30 * w) * cells
        assert bench.algorithmic_bytes("emf", n, mixed) == 8 * w * cells
    assert bench.BYTES_PER_CELL_UPDATE == 216


def test_reference_arm_prints_one_contract_line():
    if not (ROOT / "oracle" / "_ref" / "ref_cart_release_v3").exists():
        pytest.skip("oracle/_ref not built")
    # at least 3 warm-up steps (a smaller --warmup is raised to 3)
    # a 32^3 grid keeps the CPU suite short; the default is the workload's 256^3
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--n", "32"], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 3
    assert d["unit"] == "Mcell-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    # the workload's own grid, as ranks of one thread each (README mode)
    assert d["config"]["workload"] == "blast3d_periodic_32^3_fp64"
    assert d["config"]["grid"] == [32, 32, 32] and "sample_grid" not in d["config"]
    dims = d["config"]["process_grid"]
    assert d["config"]["threads_per_rank"] == 1
    assert d["config"]["ranks"] == dims[0] * dims[1] * dims[2] == d["cpu_baseline"]["cores"]


def test_rank_grid_divides_the_workload():
    import bench
    for cores in (1, 3, 8, 16, 24, 64, 112):
        for n in ((256, 256, 256), (128, 128, 128), (32, 32, 32)):
            dims = bench.rank_dims(cores, n)
            r = dims[0] * dims[1] * dims[2]
            assert r <= max(cores, 1) and all(n[a] % dims[a] == 0 for a in range(3))
