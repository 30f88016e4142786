"""The autotuner's candidate plan and selection (CPU; the measurement itself
needs a B200)."""
import json

import pytest

from cpfem_code_b200 import autotune, build


def test_every_candidate_of_every_knob_is_built():
    n = autotune.n_libs()
    for knob, cands in autotune.KNOBS.items():
        seen = [autotune.defines_of(i) for i in range(n)]
        for c in cands:
            assert any(all(d[k] == v for k, v in c.items()) for d in seen), (knob, c)


def _fake(i, us27, us81, mixed, pts, sw=(252, 318)):
    return dict(defines=autotune.defines_of(i), cube64_sweep_us=us27, cube64_sweeps=sw[0],
                brick20_32_sweep_us=us81, brick20_32_sweeps=sw[1], mixed32_cp_ms=mixed, points_cp_ms=pts,
                cube64_fp32_sweep_us=us27 / 2, cube64_fp32_sweeps=sw[0],
                brick20_32_fp32_sweep_us=us81 / 2, brick20_32_fp32_sweeps=sw[1])


def test_select_takes_the_best_candidate_per_knob(tmp_path):
    meas = {str(i): _fake(i, 130 - i, 200 + i, 10 + i, 20 - i) for i in range(autotune.n_libs())}
    # sor27 best: the last library; sor81 best: the first; cp: mixed grows, points falls
    out = tmp_path / "tuned.json"
    t = autotune.select(meas, str(out))
    sor27 = autotune.KNOBS["sor27"][len(autotune.KNOBS["sor27"]) - 1]
    sor81 = autotune.KNOBS["sor81"][0]
    for k, v in {**sor27, **sor81}.items():
        assert t["defines"][k] == v
    assert json.loads(out.read_text())["defines"] == t["defines"]


def test_select_rejects_candidates_that_change_sweep_counts(tmp_path):
    meas = {str(i): _fake(i, 120, 200, 10, 20, sw=(252 + (i == 2), 318)) for i in range(autotune.n_libs())}
    with pytest.raises(AssertionError):
        autotune.select(meas, str(tmp_path / "t.json"))


def test_build_reads_the_committed_choice():
    d = build.tuned_defines()
    if d:
        for knob, cands in autotune.KNOBS.items():
            assert any(all(d[k] == v for k, v in c.items()) for c in cands), knob


def test_select_skips_candidates_the_device_refused(tmp_path):
    """A library whose combination the device refused (recorded with an
    error) scores worst in every knob; the others are still ranked."""
    meas = {str(i): _fake(i, 130 - i, 200 + i, 10 + i, 20 - i) for i in range(autotune.n_libs())}
    last = str(autotune.n_libs() - 1)
    meas[last] = dict(defines=autotune.defines_of(int(last)), error="fas_gpu_create: ABI error -3")
    t = autotune.select(meas, str(tmp_path / "tuned.json"))
    sor27 = autotune.KNOBS["sor27"]
    # the refused library held sor27's last candidate (the best one otherwise)
    best = sor27[min(len(sor27) - 1, autotune.n_libs() - 2)]
    for k, v in best.items():
        assert t["defines"][k] == v
