"""Host-side file formats of the field export (src/analysis/export.ts:19-56)."""
import numpy as np

from windtunnel_vis_b200 import export as E


def test_js_number_strings():
    cases = {1.0: "1", 0.1: "0.1", 1e-8: "1e-8", 1.5e-7: "1.5e-7", 0.000123: "0.000123", 1e21: "1e+21",
             1e20: "100000000000000000000", -0.005: "-0.005", 2.5: "2.5", 123456800.0: "123456800"}
    for v, t in cases.items():
        assert E.js_number_string(v) == t, v


def test_csv_matches_to_precision_7():
    out = E.csv(["t", "cd"], [[1.0, 1 / 3], [2.0, float("nan")], [1e-9, "x"]], ["case sphere"])
    assert out == "# case sphere\nt,cd\n1,0.3333333\n2,\n1e-9,x\n"


def test_vtk_layout():
    dims = (3, 2, 2)
    n = 12
    rng = np.random.default_rng(0)
    f = {"dims": dims, "stride": 2, "vel": rng.random((n, 4), dtype=np.float32),
         "mean": rng.random((n, 4), dtype=np.float32), "vort": rng.random((n, 4), dtype=np.float32)}
    U, L, dx, rho_ref = 0.05, 20.0, 0.01, 1.0
    b = E.vtk(f, dx, U, L, rho_ref, "sphere")
    head = b"# vtk DataFile Version 3.0\nsphere\nBINARY\nDATASET STRUCTURED_POINTS\nDIMENSIONS 3 2 2\n" \
           b"ORIGIN 0.005 0.005 0.005\nSPACING 0.02 0.02 0.02\nPOINT_DATA 12\nVECTORS velocity float\n"
    assert b.startswith(head)
    vel = np.frombuffer(b[len(head):len(head) + n * 12], ">f4").reshape(n, 3)
    np.testing.assert_array_equal(vel, (f["vel"][:, :3].astype(np.float64) / U).astype(np.float32))
    # 3 vector and 3 scalar sections: data bytes + headers
    assert len(b) == len(head) + 3 * n * 12 + 3 * n * 4 + sum(len(s) for s in (
        b"\nVECTORS mean_velocity float\n", b"\nVECTORS vorticity float\n", b"\nSCALARS Cp float 1\nLOOKUP_TABLE default\n",
        b"\nSCALARS mean_Cp float 1\nLOOKUP_TABLE default\n", b"\nSCALARS Q_criterion float 1\nLOOKUP_TABLE default\n",
        b"\n"))
    q = np.frombuffer(b[-(n * 4 + 1):-1], ">f4")
    np.testing.assert_array_equal(q, (f["vort"][:, 3].astype(np.float64) * L * L / (U * U)).astype(np.float32))
