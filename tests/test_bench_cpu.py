"""The bench's roofline arithmetic for the persistent inner solves (no GPU).

The algorithmic bytes per row of one inner iteration restate the phases of
cgxx_b200/csrc/persist.cuh and fused.cuh (FP32 vectors 4 bytes, the band
values U 16, the factor's band Gb 8); a launch's last iteration stops after
its residual test. The roofline divides the bytes of the iterations the
timed solves ran by the device time of their persistent launches.
"""
import types

import pytest

import bench

# Bytes each phase moves per row: (reads, writes).
PHASES = {
    ("split", True): [
        ("q = A p", ["U16", "p"], ["q"]),
        ("r -= a q, d += a p", ["r", "q", "d", "p"], ["r", "d"]),
        ("y = G^T r", ["Gb8", "r"], ["y"]),
        ("z = G y + eps C r", ["Gb8", "y", "r", "C"], ["z"]),
        ("p = z + b p", ["p", "z"], ["p"]),
    ],
    # N >= 3M rows: d += a p moves into the direction phase (p read once)
    ("split-deferred", True): [
        ("q = A p", ["U16", "p"], ["q"]),
        ("r -= a q", ["r", "q"], ["r"]),
        ("y = G^T r", ["Gb8", "r"], ["y"]),
        ("z = G y + eps C r", ["Gb8", "y", "r", "C"], ["z"]),
        ("d += a p, p = z + b p", ["p", "z", "d"], ["p", "d"]),
    ],
    ("split", False): [
        ("q = A p", ["U16", "p"], ["q"]),
        ("r -= a q, d += a p, <r,Cr>", ["r", "q", "d", "p", "C"], ["r", "d"]),
        ("p = C r + b p", ["p", "r", "C"], ["p"]),
    ],
    ("fused", True): [
        ("p, d, q = A p", ["U16", "z", "p_old", "d"], ["d", "p_new", "q"]),
        ("r, y = G^T r", ["r_old", "q", "Gb8"], ["r_new", "y"]),
        ("z = G y + eps C r", ["Gb8", "y", "r", "C"], ["z"]),
    ],
    ("fused", False): [
        ("p, d, q = A p", ["U16", "z", "p_old", "d"], ["d", "p_new", "q"]),
        ("r, z = C r", ["r", "q", "C"], ["r", "z"]),
    ],
}


def _size(name):
    return {"U16": 16, "Gb8": 8}.get(name, 4)


def _bytes(phases):
    return sum(sum(_size(x) for x in rd) + sum(_size(x) for x in wr) for _, rd, wr in phases)


@pytest.mark.parametrize("form,code", [("fused", 1), ("split", 2)])
@pytest.mark.parametrize("learned", [True, False])
def test_persist_bytes_restate_the_phases(form, code, learned):
    phases = PHASES[(form, learned)]
    full, last = bench.PERSIST_BYTES[(code, learned)]
    assert full == _bytes(phases)
    # The last iteration of a launch stops after its residual test (phase B
    # of the split form, the second phase of the fused one).
    assert last == _bytes(phases[:2])


def test_deferred_split_bytes_restate_the_phases():
    phases = PHASES[("split-deferred", True)]
    full, last = bench.PERSIST_BYTES_DEFERRED[(2, True)]
    assert full == _bytes(phases)
    assert last == _bytes(phases[:2])


def test_persist_roofline_divides_the_iterations_bytes_by_the_launch_time():
    args = types.SimpleNamespace(path="learned", graph=0, n=160, stencil=7)
    N = 4_096_000
    results = [{"inner_form": 2, "fell_back": 0, "inner_launches": 3, "iterations": 330,
                "inner_ms": 24.0} for _ in range(2)]
    roof = bench.persist_roofline(args, results, N, 6530.0, "measured")
    full, last = bench.PERSIST_BYTES_DEFERRED[(2, True)]  # N >= 3M rows
    per_solve = (330 * full - 3 * (full - last)) * N
    assert roof["algorithmic_bytes"] == pytest.approx(per_solve / 3)
    assert roof["launch_us"] == pytest.approx(8000.0)
    assert roof["achieved"] == pytest.approx(per_solve / 24e-3 / 1e9)
    assert roof["frac"] == pytest.approx(roof["achieved"] / 6530.0)
    assert roof["iterations_per_launch"] == pytest.approx(110.0)


def test_persist_roofline_skips_other_forms():
    args = types.SimpleNamespace(path="learned", graph=0, n=128, stencil=27)
    r = [{"inner_form": 3, "fell_back": 0, "inner_launches": 2, "iterations": 164,
          "inner_ms": 15.0}]
    assert bench.persist_roofline(args, r, 2_097_152, 6530.0, "measured") is None
    r[0]["inner_form"] = 0
    assert bench.persist_roofline(args, r, 2_097_152, 6530.0, "measured") is None
    args.path = "plain"
    r[0]["inner_form"] = 2
    assert bench.persist_roofline(args, r, 2_097_152, 6530.0, "measured") is None


def test_persist_roofline_takes_the_undeferred_bytes_below_3m_rows():
    args = types.SimpleNamespace(path="learned", graph=0, n=128, stencil=7)
    N = 2_097_152
    r = [{"inner_form": 2, "fell_back": 0, "inner_launches": 2, "iterations": 254,
          "inner_ms": 10.0}]
    roof = bench.persist_roofline(args, r, N, 6530.0, "measured")
    full, last = bench.PERSIST_BYTES[(2, True)]
    assert roof["algorithmic_bytes"] == pytest.approx((254 * full - 2 * (full - last)) * N / 2)
