"""Initial-field tooling: coarse turbulent fields spline-interpolated to a run's grid.

Restates misc/Turb_Gen/Interpolate_Initial_Fields.m (with get_z.m) in numpy:

* coarse inputs are raw float64 files of nx1*ny1*nz1 values in Fortran order
  (x fastest), e.g. the reference's 32^3 `coarse_{u,v,w,p}_32_cubic.dat`
  (Interpolate_Initial_Fields.m:69-75); a missing input ends the loop there, as
  the script's `exist` check does (:63-67), so the absent coarse_t leaves no
  init_t.dat;
* node coordinates: x and y equispaced including both ends
  (`linspace(0, L, n)`, :28-34), z from get_z (a tanh grid with both walls as
  nodes, slope parameter 1.1, symmetric about the mid-plane, get_z.m:1-13);
* interpolation: Matlab's `interp3(..., 'spline')` on gridded data, i.e. the
  tensor product of cubic not-a-knot splines, evaluated here one axis at a time
  (the tensor-product interpolant is unique, so the axis order does not matter);
* outputs init_{u,v,w,p,t}.dat as raw float64 of the refined grid, u multiplied
  by `uscaling` (:80-85). These are the files read_init_fields reads (restart = 1,
  src/module_tools.f90:260-316); the reference stores u + u_mrf there.

The script builds its coordinate arrays with meshgrid(x, y, z) but reshapes the
data to (nx, ny, nz), so Matlab takes the data's first index as y; it then writes
the result with that first index fastest. The two agree with the x-fastest layout
that HERCULES reads only when nx2 = ny2 (and nx1 = ny1, as in the 32^3 inputs):
the default `layout="x_fastest"` writes what that case writes for any grid;
`layout="reference"` reproduces the script's byte order also when nx2 != ny2.
"""
from __future__ import annotations

import math
import os
from typing import Dict, Optional, Sequence

import numpy as np

FIELDS = ("u", "v", "w", "p", "t")


def get_z(zmin: float, zmax: float, nz: int, alpha: float = 1.1) -> np.ndarray:
    """get_z.m: nz nodes, z(1) = zmin, z(nz) = zmax, clustered at both walls."""
    zmean = 0.5 * (zmin + zmax)
    a = (1 + nz) * 0.5
    i = np.arange(1, nz + 1, dtype=np.float64)
    return zmean + (zmin - zmean) / math.tanh(2 * alpha) * np.tanh(2 * alpha * (i - a) / (1 - a))


def spline_matrix(x: np.ndarray, xq: np.ndarray) -> np.ndarray:
    """The (len(xq), len(x)) matrix W with W @ y = s(xq), s the cubic spline
    through (x, y) with not-a-knot end conditions (the third derivative is
    continuous across the second and the next-to-last node), which is Matlab's
    `spline`. Two nodes give the line, three the parabola through them."""
    x = np.asarray(x, dtype=np.float64)
    xq = np.asarray(xq, dtype=np.float64)
    n = x.size
    if n < 2:
        raise ValueError("need at least two nodes")
    if np.any(np.diff(x) <= 0):
        raise ValueError("nodes must increase")
    eye = np.eye(n)
    if n == 2:
        t = (xq - x[0]) / (x[1] - x[0])
        return np.stack([1 - t, t], axis=1)
    if n == 3:
        # the quadratic through the three nodes (Lagrange basis)
        L = np.empty((xq.size, 3))
        for j in range(3):
            o = [q for q in range(3) if q != j]
            L[:, j] = (xq - x[o[0]]) * (xq - x[o[1]]) / ((x[j] - x[o[0]]) * (x[j] - x[o[1]]))
        return L
    h = np.diff(x)
    # unknowns: second derivatives M (n). Interior rows: continuity of s'.
    A = np.zeros((n, n))
    B = np.zeros((n, n))            # right-hand side as a linear map of y
    for i in range(1, n - 1):
        A[i, i - 1] = h[i - 1]
        A[i, i] = 2.0 * (h[i - 1] + h[i])
        A[i, i + 1] = h[i]
        B[i] = 6.0 * ((eye[i + 1] - eye[i]) / h[i] - (eye[i] - eye[i - 1]) / h[i - 1])
    # not-a-knot: s''' equal on both sides of node 1 and of node n-2
    A[0, 0], A[0, 1], A[0, 2] = h[1], -(h[0] + h[1]), h[0]
    A[n - 1, n - 3], A[n - 1, n - 2], A[n - 1, n - 1] = h[n - 2], -(h[n - 3] + h[n - 2]), h[n - 3]
    Mmap = np.linalg.solve(A, B)     # M = Mmap @ y
    # evaluate on the interval of each query (end intervals extend outward)
    k = np.clip(np.searchsorted(x, xq, side="right") - 1, 0, n - 2)
    hk = h[k]
    a = (x[k + 1] - xq) / hk
    b = (xq - x[k]) / hk
    W = np.zeros((xq.size, n))
    rows = np.arange(xq.size)
    W[rows, k] += a
    W[rows, k + 1] += b
    c2 = ((a ** 3 - a) * hk ** 2 / 6.0)[:, None]
    d2 = ((b ** 3 - b) * hk ** 2 / 6.0)[:, None]
    W += c2 * Mmap[k] + d2 * Mmap[k + 1]
    return W


def interpolate(field: np.ndarray, src: Sequence[np.ndarray], dst: Sequence[np.ndarray]) -> np.ndarray:
    """Tensor-product not-a-knot spline of `field` (nz1, ny1, nx1; x fastest) from
    the node coordinates src = (x1, y1, z1) to dst = (x2, y2, z2); returns
    (nz2, ny2, nx2)."""
    f = np.asarray(field, dtype=np.float64)
    Wx = spline_matrix(src[0], dst[0])
    Wy = spline_matrix(src[1], dst[1])
    Wz = spline_matrix(src[2], dst[2])
    f = np.einsum("kji,ai->kja", f, Wx, optimize=True)
    f = np.einsum("kja,bj->kba", f, Wy, optimize=True)
    return np.einsum("kba,ck->cba", f, Wz, optimize=True)


def read_coarse(path: str, n: Sequence[int]) -> Optional[np.ndarray]:
    """A raw float64 (nx, ny, nz) Fortran-order file as (nz, ny, nx); None if absent."""
    if not os.path.exists(path):
        return None
    a = np.fromfile(path, dtype=np.float64)
    if a.size != n[0] * n[1] * n[2]:
        raise ValueError(f"{path}: {a.size} values, expected {n[0] * n[1] * n[2]}")
    return a.reshape(n[2], n[1], n[0])


def refine(coarse: Dict[str, np.ndarray], lx: float, ly: float, lz: float, n2: Sequence[int],
           uscaling: float = 1.0) -> Dict[str, np.ndarray]:
    """The refined fields ((nz2, ny2, nx2), x fastest) of the coarse ones on the
    script's node coordinates; u times uscaling."""
    out = {}
    for name, f in coarse.items():
        nz1, ny1, nx1 = f.shape
        src = (np.linspace(0.0, lx, nx1), np.linspace(0.0, ly, ny1), get_z(0.0, lz, nz1))
        dst = (np.linspace(0.0, lx, n2[0]), np.linspace(0.0, ly, n2[1]), get_z(0.0, lz, n2[2]))
        r = interpolate(f, src, dst)
        out[name] = r * uscaling if name == "u" else r
    return out


def write_init_files(results: str, lx: float, ly: float, lz: float, n1: Sequence[int], n2: Sequence[int],
                     coarse_dir: str, uscaling: float = 1.0, layout: str = "x_fastest",
                     pattern: str = "coarse_{f}_32_cubic.dat") -> Dict[str, np.ndarray]:
    """The script end to end: read coarse_{u,v,w,p,t} (stopping at the first
    missing one), refine, write init_{f}.dat under `results`. Returns the
    refined fields (nz2, ny2, nx2)."""
    os.makedirs(results, exist_ok=True)
    out = {}
    for f in FIELDS:
        c = read_coarse(os.path.join(coarse_dir, pattern.format(f=f)), n1)
        if c is None:
            break
        if layout == "x_fastest":
            r = refine({f: c}, lx, ly, lz, n2, uscaling)[f]
            r.tofile(os.path.join(results, f"init_{f}.dat"))
        elif layout == "reference":
            r = _refine_reference_layout(c, lx, ly, lz, n2, uscaling if f == "u" else 1.0)
            r.tofile(os.path.join(results, f"init_{f}.dat"))
        else:
            raise ValueError(layout)
        out[f] = r
    return out


def _refine_reference_layout(c: np.ndarray, lx, ly, lz, n2, scale):
    """The script's own result order: Matlab reads the data array's first index
    (the file's fastest, HERCULES's x) against the y nodes and its second against
    the x nodes, and writes the result with the y-node index fastest."""
    nz1, ny1, nx1 = c.shape
    nx2, ny2, nz2 = n2
    # V[p, q, r] = file value with p fastest (p along the y nodes, q along the x nodes)
    V = np.transpose(c, (2, 1, 0))                      # (nx1 = first index, ny1, nz1)
    yv1 = np.linspace(0.0, ly, V.shape[0])               # meshgrid rows: y nodes
    xv1 = np.linspace(0.0, lx, V.shape[1])
    zv1 = get_z(0.0, lz, V.shape[2])
    Wa = spline_matrix(yv1, np.linspace(0.0, ly, ny2))
    Wb = spline_matrix(xv1, np.linspace(0.0, lx, nx2))
    Wc = spline_matrix(zv1, get_z(0.0, lz, nz2))
    out = np.einsum("pqr,ap->aqr", V, Wa, optimize=True)
    out = np.einsum("aqr,bq->abr", out, Wb, optimize=True)
    out = np.einsum("abr,cr->abc", out, Wc, optimize=True)   # (ny2, nx2, nz2), a fastest on output
    return (out * scale).reshape(-1, order="F")
