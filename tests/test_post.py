"""Post-processing writers (postprocessing_functions.cpp formats) on the CPU."""
import types

import numpy as np

from memphys_b200 import post


def tiny_points(order=None):
    xyz = np.array([[0.0, 0.0], [0.5, 0.25], [1.0, 1.0 / 3.0]])
    return types.SimpleNamespace(nv=3, dim=2, xyz=xyz, order=order,
                                 boundary_flag=np.array([1, 0, 1], np.uint8))


def test_tecplot_steady_format(tmp_path):
    pts = tiny_points()
    path = post.write_tecplot_steady_variables(str(tmp_path / "run"), pts, ["u", "p"],
                                               [np.array([1.0, 2.5, -3.0]), np.array([0.1, 0.2, 0.3])],
                                               elements=[[0, 1, 2], [0, 1]])
    lines = open(path).read().splitlines()
    assert lines[0] == 'VARIABLES="x", "y", "u", "p"'      # :775-780
    assert lines[1] == ('ZONE T="1"  DATAPACKING=POINT, NODES=3, ELEMENTS=1, ZONETYPE=FETRIANGLE')
    assert lines[2] == "0 0 1 0.1 "                          # %.16g with a trailing blank
    assert lines[3] == "0.5 0.25 2.5 0.2 "
    assert lines[4] == "1 0.3333333333333333 -3 0.3 "
    assert lines[5] == "1 2 3 "                              # 1-based triangle, the edge skipped
    assert len(lines) == 6


def test_tecplot_temporal_and_reordered_points(tmp_path):
    # points renumbered by order: row i of the file is input node i, valued at order[i]
    order = np.array([2, 0, 1])
    pts = tiny_points(order)
    pts.xyz = pts.xyz.copy()
    pts.xyz[order] = tiny_points().xyz
    prefix = str(tmp_path / "run")
    post.write_tecplot_temporal_variables_header(prefix, 2, ["u"])
    u_current = np.array([10.0, 20.0, 30.0])
    post.write_tecplot_temporal_variables(prefix, pts, 0.5, ["u"], [u_current], 3)
    lines = open(prefix + "_tecplot_temporal.plt").read().splitlines()
    assert lines[0] == 'VARIABLES="x", "y", "u"'
    assert lines[1].startswith('ZONE T="1.5"  DATAPACKING=POINT, NODES=3, ELEMENTS=0')
    assert lines[2] == "0 0 30 "   # input node 0 lives at current index 2
    assert lines[3] == "0.5 0.25 10 "


def test_csv_writers(tmp_path):
    p = tmp_path / "xyz.csv"
    post.write_csv_xyz(np.array([0.0, 1.5, 2.0, -1.0]), 2, str(p))
    assert open(p).read() == "no,x,y\n0,0,1.5\n1,2,-1\n"
    q = tmp_path / "t.csv"
    post.write_csv_temporal_data_init(3, str(q))
    post.write_csv_temporal_data(np.array([1.0, 2.0, 0.125]), 0.25, str(q))
    assert open(q).read() == "time(s),0,1,2\n0.25,1,2,0.125\n"


def test_max_l1_error_split():
    a = np.array([0.0, 1.0, -3.0, 2.0])
    b = np.zeros(4)
    assert post.calc_max_l1_error(b, a) == (3.0, 1.5)
    mb, lb, mi, li = post.calc_max_l1_error(b, a, np.array([1, 0, 1, 0]))
    assert (mb, lb, mi, li) == (3.0, 1.5, 2.0, 1.5)


class _CpuCloud:
    """Operators as scipy matrices: the post-processing code only applies them."""

    def __init__(self, ops):
        self.ops = ops

    def operator(self, which):
        return self.ops[which]



def test_max_l1_error_nan_and_empty_parts():
    """general_functions.cpp:940-1032: `max_err < fabs(d)` skips NaN in the maximum, the
    mean carries it, and a part without entries divides 0 by 0."""
    a = np.array([0.0, 1.0, np.nan, 4.0])
    m, l1 = post.calc_max_l1_error(a, np.zeros(4))
    assert m == 4.0 and np.isnan(l1)
    mb, lb, mi, li = post.calc_max_l1_error(np.ones(3), np.zeros(3), np.zeros(3, bool))
    assert mb == 0.0 and np.isnan(lb) and mi == 1.0 and li == 1.0

def test_error_and_residual_tables(tmp_path):
    import scipy.sparse as sp
    from memphys_b200 import capi
    rng = np.random.default_rng(3)
    nv = 6
    gx, gy, lap = (sp.csr_matrix(rng.standard_normal((nv, nv))) for _ in range(3))
    cloud = _CpuCloud({capi.MP_GRAD_X: gx, capi.MP_GRAD_Y: gy, capi.MP_LAPLACIAN: lap})
    pts = types.SimpleNamespace(nv=nv, dim=2, boundary_flag=np.array([1, 0, 0, 1, 0, 0], np.uint8))
    u, v = rng.standard_normal(nv), rng.standard_normal(nv)
    p = np.append(rng.standard_normal(nv), 0.7)         # bordered pressure
    ua, va, pa = u + 0.01, v - 0.02, p + 5.0             # a level shift of p is no error
    e = post.calc_navier_stokes_errors_2D(pts, cloud, ua, va, pa, u, v, p)
    assert np.allclose(e["U X-vel"], (0.01, 0.01, 0.01, 0.01, 0.01, 0.01))
    assert np.allclose(e["Pressure"], 0.0, atol=1e-14)
    cont = gx @ u + gy @ v
    b = pts.boundary_flag.astype(bool)
    assert np.isclose(e["continuity"][0], np.abs(cont[~b]).max())
    path = post.write_navier_stokes_errors_2D(str(tmp_path / "r"), pts, cloud, ua, va, pa, u, v, p)
    lines = open(path).read().splitlines()
    assert lines[0] == "Errors,wrt,Analytical,solution"
    assert lines[1] == ",max_internal,avg_internal,max_boundary,avg_boundary,max_overall,avg_overall"
    assert [l.split(",")[0] for l in lines[2:]] == ["continuity", "U X-vel", "V Y-vel", "Pressure"]
    prm = types.SimpleNamespace(rho=2.0, mu=0.5)
    path = post.write_navier_stokes_residuals_2D(str(tmp_path / "r"), "_res.csv", pts, cloud, prm,
                                                 u, v, p)
    rows = open(path).read().splitlines()
    xm = u * (gx @ u) + v * (gy @ u) - 0.5 * (lap @ u) / 2.0 + (gx @ p[:nv]) / 2.0
    assert rows[3].startswith("X-mom,")
    vals = [float(x) for x in rows[3].split(",")[1:]]
    assert np.isclose(vals[4], np.abs(xm).max()) and np.isclose(vals[5], np.abs(xm).mean())


def test_iteration_details(tmp_path):
    path = post.write_iteration_details(str(tmp_path / "r"), [12, 9], [1e-9, 2.5e-9], [0.5, 0.25])
    assert open(path).read() == ("it,n_iter_actual,rel_res_log,abs_res_log\n"
                                 "0,12,1e-09,0.5\n1,9,2.5e-09,0.25\n")
    path = post.write_iteration_details(str(tmp_path / "s"), [3], [1e-9], [0.5], [0.125])
    assert open(path).read().splitlines()[1] == "0,3,1e-09,0.5,0.125"
