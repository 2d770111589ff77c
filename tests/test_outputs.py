"""The output writers reproduce the reference's files byte for byte when given the
reference's own fields (the oracle restatement is bit-exact with the reference)."""
import numpy as np
import pytest

from cfd_solver_b200.grid import ogrid
from cfd_solver_b200.outputs import parse_spt, write_coeff_his, write_spt, write_surf_dist
from oracle import refrun


@pytest.mark.skipif(not (refrun.REF_DIR / "cfd_ref").exists(),
                    reason="compiled reference not built (oracle/build_ref.sh)")
def test_writers_match_reference_files(tmp_path, oracle_lib):
    g = ogrid(24, 18, skew=0.1)
    prm = dict(Re=100.0, Ri=1.0, dt=1e-3)
    r = refrun.run(g, 1, prm)  # loop 0 writes the files
    case = oracle_lib.OracleCase(g, **prm)
    d = case.step(1)
    f = {k: case.field(k) for k in ("u", "v", "T", "p", "si", "vort")}
    write_spt(tmp_path / "spt100.dat", g, f)
    write_surf_dist(tmp_path / "SURF_DIST.dat", g, f)
    write_coeff_his(tmp_path / "COEFF_HIS.dat", int(d["time"][0]), d["cl"][0], d["cd"][0], d["cm"][0], d["nu"][0])
    write_coeff_his(tmp_path / "COEFF_HIS_pr_vor.dat", int(d["time"][0]), d["cl_pr"][0], d["cd_pr"][0],
                    d["cl_vor"][0], d["cd_vor"][0])
    for fn in ("spt100.dat", "SURF_DIST.dat", "COEFF_HIS.dat", "COEFF_HIS_pr_vor.dat"):
        assert (tmp_path / fn).read_text() == r["files"][fn], fn


def test_spt_roundtrip(tmp_path):
    g = ogrid(12, 9)
    rng = np.random.default_rng(0)
    f = {k: rng.standard_normal((g.n1, g.n0)) for k in ("u", "v", "T", "p", "si", "vort")}
    write_spt(tmp_path / "s.dat", g, f)
    back = parse_spt(tmp_path / "s.dat")
    for k in f:
        assert np.allclose(back[k], f[k], rtol=1e-12, atol=0)
