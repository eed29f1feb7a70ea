"""The cg_b200 program's drop-in surface without a GPU: usage, environment
switches and file errors give the reference's messages and exit status
(tests/golden/reference_runs.json was recorded from the reference's own
cg_serial)."""
import json
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")
EXE = os.path.join(REPO, "cgxx_b200", "cg_b200")
RUNS = json.load(open(os.path.join(GOLD, "reference_runs.json")))

pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="cg_b200 not built")


def run(args, env=None):
    e = {k: v for k, v in os.environ.items() if not k.startswith("CG_")}
    e.update(env or {})
    return subprocess.run([EXE, *args], capture_output=True, text=True, env=e, timeout=60)


def test_usage():
    p = run([])
    assert p.returncode == 1
    assert p.stderr.strip() == f"Usage: {EXE} <matrix.mtx> [<repetitions>]"
    assert run(["a", "b", "c"]).returncode == 1


@pytest.mark.parametrize("case", RUNS["errors"], ids=lambda c: c["file"] + str(c["env"]))
def test_errors_match_reference(case):
    p = run([os.path.join(GOLD, case["file"])], case["env"])
    assert p.returncode == case["rc"] == 1
    assert p.stderr.strip().splitlines()[-1] == case["stderr"]


def test_new_switch_errors():
    mtx = os.path.join(GOLD, "poisson16.mtx")
    p = run([mtx], {"CG_B200_PRECISION": "fp16"})
    assert p.returncode == 1 and "CG_B200_PRECISION" in p.stderr
    p = run([mtx], {"CG_B200_LOOP": "spin"})
    assert p.returncode == 1 and "CG_B200_LOOP" in p.stderr
    p = run([mtx], {"CG_B200_PRECISION": "mixed", "CG_PRECONDITIONER": "none"})
    assert p.returncode == 1 and "Mixed precision needs Jacobi" in p.stderr


def test_reads_matrix_before_touching_the_device():
    # File errors come first, as in the reference (its CUDA backend reads the
    # matrix in CG::init before any transfer).
    p = run([os.path.join(GOLD, "does_not_exist.mtx")])
    assert p.returncode == 1
    assert p.stderr.strip() == "Can't open file with matrix!"
    assert p.stdout.startswith("Reading matrix from")


def test_learned_switch_errors(tmp_path):
    """CG_B200_LEARNED names a weight file of the learned preconditioner; a
    missing or malformed file and the combinations the learned path cannot
    run are reported before any device work."""
    mtx = os.path.join(GOLD, "poisson16.mtx")
    weights = os.path.join(REPO, "cgxx_b200", "weights", "diffusion7.gnn")
    p = run([mtx], {"CG_B200_LEARNED": str(tmp_path / "missing.gnn")})
    assert p.returncode == 1 and "Could not open weight file" in p.stderr
    bad = tmp_path / "bad.gnn"
    bad.write_bytes(open(weights, "rb").read()[:-4])  # one parameter short
    p = run([mtx], {"CG_B200_LEARNED": str(bad)})
    assert p.returncode == 1 and "Invalid weight file" in p.stderr
    p = run([mtx], {"CG_B200_LEARNED": mtx})
    assert p.returncode == 1 and "Invalid weight file" in p.stderr
    p = run([mtx], {"CG_B200_LEARNED": weights, "CG_B200_PRECISION": "fp64"})
    assert p.returncode == 1 and "runs in mixed precision" in p.stderr
    for env in ({"CG_B200_FUSED": "0"}, {"CG_PRECONDITIONER": "none"}):
        p = run([mtx], dict(env, CG_B200_LEARNED=weights))
        assert p.returncode == 1 and "needs Jacobi and the fused solve" in p.stderr
