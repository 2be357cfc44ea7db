"""The command-line driver (pbh_b200.pm3d_peak, the counterpart of pbhgr/scripts/pm3d_peak.py)
on a small run: JSON output with the reference's keys, rows at the diagnostic cadence and at
the end, and the run's last row matching `analyse` of the final state."""
import json

import pytest

pytestmark = pytest.mark.gpu


def test_driver_writes_reference_json(tmp_path):
    from pbh_b200 import pm3d_peak
    out = pm3d_peak.main(["--mu", "0.3", "--N", "16", "--Np", "16", "--L", "8", "--tend", "3",
                          "--smooth", "1", "--da_frac", "0.05", "--out", str(tmp_path)])
    path = tmp_path / (pm3d_peak.tag_of(pm3d_peak.parse(["--mu", "0.3", "--N", "16", "--Np", "16", "--L", "8",
                                                          "--tend", "3", "--smooth", "1", "--da_frac", "0.05"]))
                       + ".json")
    data = json.loads(path.read_text())
    assert set(data) == {"args", "rows", "rm", "t_H", "tC0", "dx", "m_part"}
    rows = data["rows"]
    assert len(rows) >= 3
    assert rows[-1]["t_over_tH"] == pytest.approx(3.0, rel=1e-9)
    ts = [r["t_over_tH"] for r in rows]
    assert all(b > a for a, b in zip(ts, ts[1:]))
    for key in ("axes_com_0.1", "hoop_0.2", "m_in_1c", "C_2c", "delta_max", "rho_max_over_mean", "step"):
        assert key in rows[-1]
    assert out["rm"] == pytest.approx(6 ** 0.5)
