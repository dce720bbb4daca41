"""Python access to the oracle: the C restatement (oracle/liboracle.so) and the
reference's own operators (oracle/_ref/ref_harness_{f64,f32}).

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py import this module,
and only as the checker or as the timed CPU baseline.  The product
(``gliomasolver_b200``) never imports it.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
LAB_GHOSTS = 488

_lib = None


def build_port() -> Path:
    """Compile the C restatement (``make -C oracle port``)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    return HERE / "liboracle.so"


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build_port()
        _lib = ctypes.CDLL(str(path))
        _declare(_lib)
    return _lib


class GhostCSR(ctypes.Structure):
    _fields_ = [
        ("nrows", ctypes.c_int64),
        ("row_ptr", ctypes.c_void_p),
        ("src", ctypes.c_void_p),
        ("w0", ctypes.c_void_p),
        ("w1", ctypes.c_void_p),
        ("w2", ctypes.c_void_p),
    ]


def _declare(L):
    P = ctypes.c_void_p
    I, I64, D, F = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_float
    L.orc_rd_rhs_dense_f64.argtypes = [I, P, P, P, D, D, D, D, P]
    L.orc_rd_rhs_dense_f32.argtypes = [I, P, P, P, F, F, F, F, P]
    L.orc_rd_steps_dense_f64.argtypes = [I, P, P, P, D, D, D, D, D, I, P]
    L.orc_rd_steps_dense_f32.argtypes = [I, P, P, P, F, F, F, F, D, I, P]
    L.orc_fill_ghosts_f64.argtypes = [P, P, P]
    L.orc_fill_ghosts_f32.argtypes = [P, P, P]
    L.orc_rd_rhs_pool_f64.argtypes = [I, P, P, P, P, P, P, P, D, D, D, P]
    L.orc_rd_rhs_pool_f32.argtypes = [I, P, P, P, P, P, P, P, F, F, F, P]
    L.orc_update_f64.argtypes = [I64, P, P, D]
    L.orc_update_f32.argtypes = [I64, P, P, D]
    L.orc_fwt_detail_pool_f64.argtypes = [I, P, P, P]
    L.orc_fwt_detail_pool_f32.argtypes = [I, P, P, P]
    L.orc_split_block_f64.argtypes = [P, P, P]
    L.orc_split_block_f32.argtypes = [P, P, P]
    L.orc_collapse_blocks_f64.argtypes = [P, P]
    L.orc_collapse_blocks_f32.argtypes = [P, P]
    L.orc_uq_dump_f64.argtypes = [I, P, P, P, P, I, P]
    L.orc_uq_dump_f32.argtypes = [I, P, P, P, P, I, P]
    L.orc_adjoint_step_dense_f64.argtypes = [I, P, P, P, D, D, D, D, D, P, P, P]
    L.orc_loss_grad_f64.argtypes = [I64, P, P, P, D, D, D, P]
    L.orc_map_anatomy_f64.argtypes = [I, I, I, I, P, P, P, P, P, P, P, P, P]
    L.orc_map_anatomy_f32.argtypes = [I, I, I, I, P, P, P, P, P, P, P, P, P]
    L.orc_log_likelihood.argtypes = [I, P, P, P, P, P, I, D, D, D, D, D, I, I, P]


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


def _sfx(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


# ---------------------------------------------------------------- dense grid
def rd_rhs_dense(pw, pg, phi, Dw, Dg, rho, h):
    R = pw.dtype.type
    out = np.empty_like(phi)
    getattr(lib(), "orc_rd_rhs_dense_" + _sfx(R))(
        phi.shape[0], _p(pw), _p(pg), _p(phi), R(Dw), R(Dg), R(rho), R(h), _p(out))
    return out


def rd_steps_dense(pw, pg, phi, Dw, Dg, rho, h, dt, nsteps):
    """``nsteps`` reference steps on a dense periodic grid; returns the new phi."""
    R = pw.dtype.type
    out = np.array(phi, copy=True)
    scratch = np.empty_like(phi)
    getattr(lib(), "orc_rd_steps_dense_" + _sfx(R))(
        phi.shape[0], _p(pw), _p(pg), _p(out), R(Dw), R(Dg), R(rho), R(h), float(dt),
        int(nsteps), _p(scratch))
    return out


# ---------------------------------------------------------------- block pool
def fill_ghosts(csr: dict, field: np.ndarray):
    g = GhostCSR(csr["row_ptr"].size - 1, _p(csr["row_ptr"]).value, _p(csr["src"]).value,
                 _p(csr["w0"]).value, _p(csr["w1"]).value, _p(csr["w2"]).value)
    out = np.empty(csr["row_ptr"].size - 1, dtype=field.dtype)
    getattr(lib(), "orc_fill_ghosts_" + _sfx(field.dtype))(ctypes.byref(g), _p(field), _p(out))
    return out


def rd_rhs_pool(h, pw, pg, phi, gpw, gpg, gphi, Dw, Dg, rho):
    R = pw.dtype.type
    nb = pw.size // 512
    out = np.empty_like(phi)
    getattr(lib(), "orc_rd_rhs_pool_" + _sfx(R))(
        nb, _p(np.ascontiguousarray(h, dtype=R)), _p(pw), _p(pg), _p(phi), _p(gpw), _p(gpg),
        _p(gphi), R(Dw), R(Dg), R(rho), _p(out))
    return out


def update(phi, dphidt, dt):
    out = np.array(phi, copy=True)
    getattr(lib(), "orc_update_" + _sfx(phi.dtype))(out.size, _p(out), _p(dphidt), float(dt))
    return out


def fwt_detail_pool(phi, gphi):
    nb = phi.size // 512
    out = np.empty(nb, dtype=np.float64)
    getattr(lib(), "orc_fwt_detail_pool_" + _sfx(phi.dtype))(nb, _p(phi), _p(gphi), _p(out))
    return out


def split_block(parent, gparent):
    out = np.empty(8 * 512, dtype=parent.dtype)
    getattr(lib(), "orc_split_block_" + _sfx(parent.dtype))(_p(parent), _p(gparent), _p(out))
    return out


def collapse_blocks(children):
    out = np.empty(512, dtype=children.dtype)
    getattr(lib(), "orc_collapse_blocks_" + _sfx(children.dtype))(_p(children), _p(out))
    return out


def uq_dump(levels, indices, h, phi_pool, gpd):
    """_dumpUQoutput of blocks (level, index (3,), h in Real) with phi in block order."""
    R = phi_pool.dtype.type
    lv = np.ascontiguousarray(levels, dtype=np.int32)
    ix = np.ascontiguousarray(indices, dtype=np.int32).reshape(-1)
    hh = np.ascontiguousarray(h, dtype=R)
    out = np.empty((gpd, gpd, gpd), dtype=np.float64)
    getattr(lib(), "orc_uq_dump_" + _sfx(R))(lv.size, _p(lv), _p(ix), _p(hh),
                                              _p(np.ascontiguousarray(phi_pool)), gpd, _p(out))
    return out


def log_likelihood(model, t1c, flair, pet=None, roi=None, pet_sigma2=0.000361, pet_scale=0.85, t1_uc=0.7,
                   t2_uc=0.25, slope=2.0, step_pet=1, step_mri=1):
    """HGG_Likelihood in long double; returns [L_PET, L_T1c, L_FLAIR] as float64."""
    n = model.shape[0]
    out = (ctypes.c_longdouble * 3)()
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (model, t1c, flair)]
    pe = None if pet is None else np.ascontiguousarray(pet, dtype=np.float64)
    ro = None if roi is None else np.ascontiguousarray(roi, dtype=np.int32).reshape(-1)
    lib().orc_log_likelihood(n, _p(a[0]), _p(a[1]), _p(a[2]), None if pe is None else _p(pe),
                             None if ro is None else _p(ro), 0 if ro is None else ro.size // 3,
                             pet_sigma2, pet_scale, t1_uc, t2_uc, slope, step_pet, step_mri, out)
    return np.array([float(out[0]), float(out[1]), float(out[2])])


def adjoint_dense(pw, pg, phi0, Dw, Dg, rho, h, dt, nsteps, lam_final, magnitudes=False):
    """The discrete adjoint of nsteps FP64 steps (orc_adjoint_step_dense_f64,
    every state stored): returns (dL/dphi0, dL/drho, dL/dDw) for a loss whose
    gradient with respect to the final state is lam_final; with magnitudes
    also the sums of the magnitudes of the dL/drho and dL/dDw terms."""
    L = lib()
    n = phi0.shape[0]
    pw, pg = (np.ascontiguousarray(a, dtype=np.float64) for a in (pw, pg))
    states = [np.ascontiguousarray(phi0, dtype=np.float64)]
    for _ in range(nsteps):
        states.append(rd_steps_dense(pw, pg, states[-1], Dw, Dg, rho, h, dt, 1))
    lam = np.array(lam_final, dtype=np.float64, copy=True)
    grad = np.zeros(4)
    scratch = np.empty(8 * n ** 3)
    for k in range(nsteps - 1, -1, -1):
        L.orc_adjoint_step_dense_f64(n, _p(pw), _p(pg), _p(states[k]), float(Dw), float(Dg), float(rho), float(h),
                                     float(dt), _p(lam), _p(grad), _p(scratch))
    if magnitudes:
        return lam, float(grad[0]), float(grad[1]), float(grad[2]), float(grad[3])
    return lam, float(grad[0]), float(grad[1])


def loss_grad(u, t1c, flair, t1uc=0.7, t2uc=0.25, slope=2.0):
    """d(-(L_T1c + L_FLAIR))/du (orc_loss_grad_f64)."""
    u, t1c, flair = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, t1c, flair))
    out = np.empty_like(u)
    lib().orc_loss_grad_f64(u.size, _p(u), _p(t1c), _p(flair), float(t1uc), float(t2uc), float(slope), _p(out))
    return out


def map_anatomy(gm, wm, csf, bpd, tumor_ic, precision="f64"):
    """Glioma_ReactionDiffusion::_ic restated (orc_map_anatomy_*): dense
    (8 bpd)^3 arrays p_w, p_g, p_csf, phi, tissue in the precision's Real."""
    vols = [np.ascontiguousarray(v, dtype=np.float64) for v in (gm, wm, csf)]
    sz, sy, sx = vols[0].shape
    dtype = np.float64 if precision == "f64" else np.float32
    n = 8 * int(bpd)
    outs = [np.zeros((n, n, n), dtype=dtype) for _ in range(5)]
    tic = np.ascontiguousarray(tumor_ic, dtype=np.float64)
    getattr(lib(), f"orc_map_anatomy_{precision}")(int(bpd), sx, sy, sz, *(_p(v) for v in vols), _p(tic),
                                                    *(_p(o) for o in outs))
    return dict(zip(("p_w", "p_g", "p_csf", "phi", "tissue"), outs))


# ------------------------------------------------- the reference's own code
def ref_available(precision: str = "f64") -> bool:
    return (REF_DIR / f"ref_harness_{precision}").exists()


def _write_dense(path, pw, pg, phi):
    n = pw.shape[0]
    with open(path, "wb") as f:
        f.write(np.int32(n).tobytes())
        for a in (pw, pg, phi):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())


def _fmt(x: float) -> str:
    return repr(float(x))


def ref_uniform(pw, pg, phi, Dw, Dg, rho, dt, nsteps, precision="f64", threads=None):
    """Run ``nsteps`` steps of the reference's own operators on a uniform grid."""
    n = pw.shape[0]
    env = dict(os.environ)
    if threads:
        env["GBFK_TBB_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        _write_dense(fin, pw, pg, phi)
        subprocess.run([str(REF_DIR / f"ref_harness_{precision}"), "uniform", fin, fout,
                        _fmt(Dw), _fmt(Dg), _fmt(rho), _fmt(dt), str(int(nsteps))],
                       check=True, env=env)
        return np.fromfile(fout, dtype=np.float64).reshape(n, n, n)


def ref_rhs(pw, pg, phi, Dw, Dg, rho, precision="f64"):
    n = pw.shape[0]
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        _write_dense(fin, pw, pg, phi)
        subprocess.run([str(REF_DIR / f"ref_harness_{precision}"), "rhs", fin, fout,
                        _fmt(Dw), _fmt(Dg), _fmt(rho)], check=True)
        return np.fromfile(fout, dtype=np.float64).reshape(n, n, n)


def ref_time(pw, pg, phi, Dw, Dg, rho, dt, nsteps, precision="f32", threads=None, warmup=0):
    """Time the reference's stepping loop (after ``warmup`` untimed steps);
    returns its JSON record."""
    env = dict(os.environ)
    if threads:
        env["GBFK_TBB_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        _write_dense(fin, pw, pg, phi)
        r = subprocess.run([str(REF_DIR / f"ref_harness_{precision}"), "time", fin,
                            _fmt(Dw), _fmt(Dg), _fmt(rho), _fmt(dt), str(int(nsteps)), str(int(warmup))],
                           check=True, env=env, capture_output=True, text=True)
        return json.loads(r.stdout.strip().splitlines()[-1])


def write_matrix3d(path, a):
    """The reference's Matrix .dat layout (Glioma/Matrix.h:609-631):
    int32 {1234, 3, nx, ny, nz}, int32 type id (0 = double), data x fastest."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    nz, ny, nx = a.shape
    with open(path, "wb") as f:
        f.write(np.array([1234, 3, nx, ny, nz, 0], dtype=np.int32).tobytes())
        f.write(a.tobytes())


def write_matrix2d(path, points):
    """Matrix::D2D layout with nx = number of points and ny = 3, so that
    element (i, j) = coordinate j of point i (HGG_Likelihood.cpp:108-115)."""
    a = np.ascontiguousarray(points, dtype=np.float64)
    npts, ncoord = a.shape
    with open(path, "wb") as f:
        f.write(np.array([1234, 2, npts, ncoord, 0], dtype=np.int32).tobytes())
        f.write(np.ascontiguousarray(a.T).tobytes())


def ref_likelihood(model, t1c, flair, pet, roi=None, pet_sigma2=0.000361, pet_scale=0.85, t1_uc=0.7, t2_uc=0.25,
                   slope=2.0, step_pet=1, step_mri=1):
    """Run the reference's likelihood program; returns -log-likelihood as
    written to Likelihood.txt (printed with %Lf, 6 decimals) and its stdout."""
    exe = REF_DIR / "likelihood"
    with tempfile.TemporaryDirectory() as td:
        write_matrix3d(os.path.join(td, "HGG_data.dat"), model)
        write_matrix3d(os.path.join(td, "tumT1c.dat"), t1c)
        write_matrix3d(os.path.join(td, "tumFLAIR.dat"), flair)
        write_matrix3d(os.path.join(td, "tumPET.dat"), pet)
        if roi is not None:
            write_matrix2d(os.path.join(td, "ROI.dat"), np.asarray(roi, dtype=np.float64).reshape(-1, 3))
        with open(os.path.join(td, "LikelihoodInput.txt"), "w") as f:
            f.write(f"{pet_sigma2!r}\n{pet_scale!r}\n{t1_uc!r}\n{t2_uc!r}\n{slope!r}\n")
        args = [str(exe), "-stepPET", str(step_pet), "-stepMRI", str(step_mri), "-bROI", "1" if roi is not None else "0"]
        r = subprocess.run(args, cwd=td, check=True, capture_output=True, text=True)
        with open(os.path.join(td, "Likelihood.txt")) as f:
            return float(f.read().split()[0]), r.stdout


def ref_ic_available(precision: str = "f64") -> bool:
    return (REF_DIR / f"ic_harness_{precision}").exists()


def ref_map_anatomy(prefix, bpd, tumor_ic, precision="f64"):
    """Run the reference's own Glioma_ReactionDiffusion::_ic on
    {prefix}GM.dat, WM.dat, CSF.dat (oracle/_ref/ic_harness_*).  Returns a
    dict with L, p_w, p_g, p_csf, phi (float64 copies of the Real cells) and
    the seconds _ic took."""
    n = 8 * int(bpd)
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "ic.bin")
        r = subprocess.run([str(REF_DIR / f"ic_harness_{precision}"), os.fspath(prefix), str(int(bpd)),
                            *(_fmt(v) for v in tumor_ic), out], check=True, capture_output=True, text=True)
        rec = json.loads(r.stdout.strip().splitlines()[-1])
        raw = np.fromfile(out, dtype=np.float64)
    n3 = n ** 3
    res = {"L": float(raw[0]), "seconds": rec["ic_seconds"]}
    for k, name in enumerate(("p_w", "p_g", "p_csf", "phi")):
        res[name] = raw[1 + k * n3:1 + (k + 1) * n3].reshape(n, n, n)
    return res


def ref_topology_available(precision: str = "f64") -> bool:
    return (REF_DIR / f"topo_harness_{precision}").exists()


def read_topology_dump(path) -> dict:
    """The records of oracle/_ref/topo_harness_*: int32 name length, name,
    int32 kind (0 int64, 1 float64), int64 count, data."""
    out = {}
    with open(path, "rb") as f:
        while True:
            head = f.read(4)
            if not head:
                break
            name = f.read(int(np.frombuffer(head, np.int32)[0])).decode()
            kind = int(np.frombuffer(f.read(4), np.int32)[0])
            count = int(np.frombuffer(f.read(8), np.int64)[0])
            out[name] = np.frombuffer(f.read(8 * count), np.int64 if kind == 0 else np.float64).copy()
    return out


def ref_topology(base_bpd, maxlevel, refine_tol, every, precision="f64"):
    """The reference's wavelet details, block split and collapse on an
    adapted grid (oracle/_ref/topo_harness_*, one host thread so that the
    grid is reproducible): a dict of the dump's arrays and the JSON summary
    under "summary"."""
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "topo.bin")
        r = subprocess.run([str(REF_DIR / f"topo_harness_{precision}"), str(int(base_bpd)), str(int(maxlevel)),
                            _fmt(refine_tol), str(int(every)), out], check=True, capture_output=True, text=True,
                           env=dict(os.environ, GBFK_TBB_THREADS="1"))
        res = read_topology_dump(out)
    res["summary"] = json.loads(r.stdout.strip().splitlines()[-1])
    return res


def read_matrix3d(path) -> np.ndarray:
    """A Matrix .dat of doubles as written by MatrixD3D::dump (the layout of
    write_matrix3d): shape (nz, ny, nx)."""
    raw = Path(path).read_bytes()
    head = np.frombuffer(raw[:24], dtype=np.int32)
    if head[0] != 1234 or head[1] != 3 or head[5] != 0:
        raise ValueError(f"{path}: not a 3-D Matrix of doubles")
    nx, ny, nz = (int(v) for v in head[2:5])
    return np.frombuffer(raw[24:], dtype=np.float64, count=nx * ny * nz).reshape(nz, ny, nx).copy()


def ref_uq_available(precision: str = "f64") -> bool:
    return (REF_DIR / f"uq_harness_{precision}").exists()


def ref_uq_dump(prefix, tumor_ic, refine_tol, compress_tol, precision="f64", sigma=0.0):
    """The reference's _dumpUQoutput of its own grid after _ic on
    {prefix}GM.dat, WM.dat, CSF.dat (phi replaced by a Gaussian of width
    sigma at the tumour centre when sigma > 0) and one AutomaticRefinement
    and AutomaticCompression (oracle/_ref/uq_harness_*).  Returns the leaves
    (level, index, h, phi in block order), the dump as (gpd, gpd, gpd) and
    the JSON summary."""
    with tempfile.TemporaryDirectory() as td:
        r = subprocess.run([str(REF_DIR / f"uq_harness_{precision}"), os.fspath(prefix),
                            *(_fmt(v) for v in tumor_ic), _fmt(refine_tol), _fmt(compress_tol), td, _fmt(sigma)],
                           check=True, capture_output=True, text=True, env=dict(os.environ, GBFK_TBB_THREADS="1"))
        res = read_topology_dump(os.path.join(td, "leaves.bin"))
        res["dump"] = read_matrix3d(os.path.join(td, "HGG_data.dat"))
    res["summary"] = json.loads(r.stdout.strip().splitlines()[-1])
    return res
