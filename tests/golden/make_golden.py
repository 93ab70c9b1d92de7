"""Regenerate ref_tables.json from the reference's own sympy-generated tables.

The reference's GLL / Lagrange / simplex tables (src/cxx/Element/*/Autogen/*.c)
compile standalone; `make -C oracle` builds them into
oracle/_ref/libsalvus_ref_tables.so from the reference sources.  This script
evaluates them and writes the golden fixture that pins the oracle (and, through
the oracle, the CUDA path):

  quad orders 1..10 : GLL points, weights, closure map, derivative matrix
                      D[i][j] = l_j'(xi_i) as assembled by
                      TensorQuad::setupGradientOperator (TensorQuad.cpp:107-142),
                      tensor Lagrange values and eps/eta derivatives at sample
                      points (interpolate_orderN_square)
  hex orders 1..6   : tensor Lagrange values and r/s/t derivatives at sample
                      points (interpolate_*_orderN_hex)
  P3 triangle / tet : node coordinates, quadrature weights, dphi tables

Usage:  make -C oracle && python tests/golden/make_golden.py
"""
import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "..", "oracle", "_ref", "libsalvus_ref_tables.so")

# Sample reference coordinates (seeded, fixed) at which the tensor tables are
# evaluated; they avoid the GLL nodes so the values are non-trivial.
rng = np.random.default_rng(20160212)
SAMPLES_2D = rng.uniform(-1, 1, size=(6, 2)).round(6).tolist()
SAMPLES_3D = rng.uniform(-1, 1, size=(4, 3)).round(6).tolist()

D = ctypes.c_double
DP = ctypes.POINTER(ctypes.c_double)


def arr(n):
    return (ctypes.c_double * n)()


def main():
    lib = ctypes.CDLL(LIB)
    out = {"source": "reference sympy-generated Autogen tables", "quad": {}, "hex": {}}
    for N in range(1, 11):
        n = N + 1
        P = n * n
        pts, wts = arr(n), arr(n)
        getattr(lib, f"gll_coordinates_order{N}_square")(pts)
        getattr(lib, f"gll_weights_order{N}_square")(wts)
        cm = (ctypes.c_int * P)()
        getattr(lib, f"closure_mapping_order{N}_square")(cm)
        eps_d = getattr(lib, f"interpolate_eps_derivative_order{N}_square")
        eta_d = getattr(lib, f"interpolate_eta_derivative_order{N}_square")
        interp = getattr(lib, f"interpolate_order{N}_square")
        interp.argtypes = [D, D, DP]
        if N == 1:
            eps_d.argtypes = [D, DP]
            eta_d.argtypes = [D, DP]
        else:
            eps_d.argtypes = [D, D, DP]
            eta_d.argtypes = [D, D, DP]
        # mGrd row i = first n entries of d/d eps at (xi_i, xi_0)
        grad = []
        for i in range(n):
            t = arr(P)
            if N == 1:
                eps_d(pts[0], t)
            else:
                eps_d(pts[i], pts[0], t)
            grad.append([t[j] for j in range(n)])
        samples = []
        for (r, s) in SAMPLES_2D:
            v, dr, ds = arr(P), arr(P), arr(P)
            interp(r, s, v)
            if N == 1:
                eps_d(s, dr)
                eta_d(r, ds)
            else:
                eps_d(r, s, dr)
                eta_d(r, s, ds)
            samples.append({"ref": [r, s], "l": list(v), "dr": list(dr), "ds": list(ds)})
        out["quad"][str(N)] = {
            "points": list(pts), "weights": list(wts), "closure": list(cm),
            "grad": grad, "samples": samples,
        }
    for N in range(1, 7):
        n = N + 1
        P = n * n * n
        interp = getattr(lib, f"interpolate_order{N}_hex")
        interp.argtypes = [D, D, D, DP]
        der = [getattr(lib, f"interpolate_{c}_derivative_order{N}_hex") for c in "rst"]
        for f in der:
            f.argtypes = [D, D, DP] if N == 1 else [D, D, D, DP]
        samples = []
        for (r, s, t) in SAMPLES_3D:
            v = arr(P)
            interp(r, s, t, v)
            ds = []
            for k, f in enumerate(der):
                o = arr(P)
                if N == 1:
                    args = [(s, t), (r, t), (r, s)][k]
                    f(args[0], args[1], o)
                else:
                    f(r, s, t, o)
                ds.append(list(o))
            samples.append({"ref": [r, s, t], "l": list(v), "dr": ds[0], "ds": ds[1], "dt": ds[2]})
        out["hex"][str(N)] = {"samples": samples}
    # P3 triangle (12 nodes) and tetrahedron (50 nodes)
    tri = {}
    rn, sn, w = arr(12), arr(12), arr(12)
    lib.coordinates_p3_triangle_rn(rn)
    lib.coordinates_p3_triangle_sn(sn)
    lib.quadrature_weights_p3_triangle(w)
    dr, ds = arr(144), arr(144)
    lib.dphi_dr_rsn_p3_triangle(dr)
    lib.dphi_ds_rsn_p3_triangle(ds)
    tri.update(r=list(rn), s=list(sn), w=list(w), dphi_dr=list(dr), dphi_ds=list(ds))
    out["tri_p3"] = tri
    tet = {}
    rn, sn, tn, w = arr(50), arr(50), arr(50), arr(50)
    lib.coordinates_p3_tetrahedra_rn(rn)
    lib.coordinates_p3_tetrahedra_sn(sn)
    lib.coordinates_p3_tetrahedra_tn(tn)
    lib.quadrature_weights_p3_tetrahedra(w)
    dr, ds, dt = arr(2500), arr(2500), arr(2500)
    lib.dphi_dr_rstn_p3_tetrahedra(dr)
    lib.dphi_ds_rstn_p3_tetrahedra(ds)
    lib.dphi_dt_rstn_p3_tetrahedra(dt)
    tet.update(r=list(rn), s=list(sn), t=list(tn), w=list(w),
               dphi_dr=list(dr), dphi_ds=list(ds), dphi_dt=list(dt))
    out["tet_p3"] = tet
    with open(os.path.join(HERE, "ref_tables.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
