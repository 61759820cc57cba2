"""Python host mirror of the B200 pseudospectral step (ctypes over the C ABI).

The operator surface follows the reference solver (mfkiwl/gnss-1):
``forward_transform`` / ``inverse_transform`` (fftfuncs.cu:288-359),
``de_alias``, ``vorticity``, ``gradient``, ``divergence``, ``make_rhs``,
``timestep``, ``update``, ``cross_product``, ``dot_product``,
``colloid_advection`` and ``solver_ps`` (solver.cu), and the spectral
statistics of statistics.cu:1494-1845.  Buffers are device memory in the
reference layouts (spectral complex [ny][nx][nz2], physical real padded
[nx][ny][2*nz2], one buffer per field, transforms in place).

Arguments may be torch CUDA tensors or raw device pointers (ints).  Every call
raises :class:`GnssError` on a non-zero status.  The shared library must be
built (``python gnss-1_b200/build.py``); importing this module on a machine
where it is missing raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path
from typing import Iterable, Sequence

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libgnss_b200.so"

GNSS_OK = 0
GNSS_SCHEME_CNAB2 = 0
GNSS_SCHEME_RK3IF = 1
GNSS_FP64 = 0
GNSS_FP32 = 1
GNSS_NSTATS = 7
GNSS_OPT_ZVARIANT = 0
GNSS_OPT_PVARIANT = 1
GNSS_OPT_ZKERNEL = 2   # read-only: the z kernel the options select
GNSS_OPT_TEST_WAIT = 3  # test of the bounded device waits: poll cap, first copy of block 0 withheld (0 = off)
GNSS_ERR_TIMEOUT = 5
GNSS_VARIANT_AUTO = GNSS_ZVARIANT_AUTO = 0
GNSS_VARIANT_REGISTER = GNSS_ZVARIANT_REGISTER = 1
GNSS_VARIANT_STAGED = GNSS_ZVARIANT_STAGED = 2
GNSS_VARIANT_WARPSPEC = 3   # GNSS_OPT_ZVARIANT only
GNSS_VARIANT_TENSOR = 4     # GNSS_OPT_PVARIANT only: split-TF32 DFT-GEMM passes on tcgen05 (FP32, N = 256, 512)
STAT_NAMES = ("ke", "vrms2", "eps", "chi_s", "chi_c", "var_s", "var_c")
SUPPORTED_SIZES = (8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512)


class GnssError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        super().__init__(f"{what}: status {status}" + (f" ({detail})" if detail else ""))
        self.status = status


class GnssConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("re", ctypes.c_double), ("sc", ctypes.c_double), ("sc_c", ctypes.c_double),
        ("alpha", ctypes.c_double), ("dt", ctypes.c_double),
        ("alias_filter", ctypes.c_double), ("nu_stats", ctypes.c_double),
        ("n_scalars", ctypes.c_int), ("scheme", ctypes.c_int), ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class GnssTurb(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("vrms", "ke", "epsilon", "eta", "l", "lambda_", "chi", "omega",
                                               "omega_x", "omega_y", "omega_z")]


class GnssJetParams(ctypes.Structure):
    _fields_ = [("h", ctypes.c_double), ("theta", ctypes.c_double), ("theta_c", ctypes.c_double),
                ("pert_amp", ctypes.c_double), ("seed", ctypes.c_uint)]


class GnssFields(ctypes.Structure):
    _fields_ = [("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("w", ctypes.c_void_p),
                ("s", ctypes.c_void_p), ("c", ctypes.c_void_p)]


# name -> argtypes (all return gnss_status unless listed in _RESTYPES)
_VP = ctypes.c_void_p
_SIGS = {
    "gnss_create": [ctypes.POINTER(GnssConfig), ctypes.POINTER(ctypes.c_void_p)],
    "gnss_destroy": [_VP],
    "gnss_field_bytes": [_VP],
    "gnss_workspace_bytes": [_VP],
    "gnss_status_string": [ctypes.c_int],
    "gnss_last_error": [_VP],
    "gnss_forward": [_VP, _VP, _VP],
    "gnss_inverse": [_VP, _VP, _VP],
    "gnss_dealias": [_VP, _VP, _VP],
    "gnss_vorticity": [_VP] + [_VP] * 6 + [_VP],
    "gnss_gradient": [_VP] + [_VP] * 4 + [_VP],
    "gnss_divergence": [_VP] + [_VP] * 4 + [_VP],
    "gnss_make_rhs": [_VP] + [_VP] * 5 + [_VP],
    "gnss_timestep": [_VP, ctypes.c_int, ctypes.POINTER(GnssFields), ctypes.POINTER(GnssFields),
                      ctypes.POINTER(GnssFields), _VP],
    "gnss_update": [_VP, ctypes.POINTER(GnssFields), ctypes.POINTER(GnssFields), _VP],
    "gnss_cross_product": [_VP] + [_VP] * 6 + [_VP],
    "gnss_dot_product": [_VP] + [_VP] * 7 + [_VP],
    "gnss_colloid_advection": [_VP] + [_VP] * 11 + [_VP],
    "gnss_step": [_VP, ctypes.POINTER(GnssFields), ctypes.POINTER(GnssFields), ctypes.c_int, _VP],
    "gnss_stats": [_VP, ctypes.POINTER(GnssFields), ctypes.POINTER(ctypes.c_double), _VP],
    "gnss_run_host": [_VP, _VP, _VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _VP],
    "gnss_run_host_bytes": [_VP, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)],
    "gnss_launch_count": [_VP],
    "gnss_check": [_VP, _VP],
    "gnss_forward_noalloc": [ctypes.POINTER(GnssConfig), _VP, _VP],
    "gnss_profile_enable": [_VP, ctypes.c_int],
    "gnss_stage_bytes": [_VP, ctypes.POINTER(ctypes.c_double)],
    "gnss_set_option": [_VP, ctypes.c_int, ctypes.c_int],
    "gnss_get_option": [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)],
    "gnss_profile_read": [_VP, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)],
    "gnss_scratch_bytes": [_VP],
    "gnss_initial_jet": [_VP, ctypes.POINTER(GnssJetParams), ctypes.POINTER(GnssFields), _VP],
    "gnss_get_config": [_VP, ctypes.POINTER(GnssConfig)],
    "gnss_io_write_field": [ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP, ctypes.c_char_p],
    "gnss_io_read_field": [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, _VP],
    "gnss_io_write_slice": [ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP, ctypes.c_int, ctypes.c_int,
                            ctypes.c_char_p],
    "gnss_io_write_stat": [ctypes.c_char_p, ctypes.c_double, ctypes.c_int],
    "gnss_io_write_profile": [ctypes.c_int, _VP, ctypes.c_char_p],
    "gnss_save_state": [_VP, ctypes.POINTER(GnssFields), ctypes.c_char_p, ctypes.c_int, _VP],
    "gnss_load_state": [_VP, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(GnssFields), _VP],
    "gnss_checkpoint_save": [_VP, ctypes.POINTER(GnssFields), ctypes.POINTER(GnssFields), ctypes.c_longlong,
                             ctypes.c_char_p, _VP],
    "gnss_checkpoint_load": [_VP, ctypes.c_char_p, ctypes.POINTER(GnssFields), ctypes.POINTER(GnssFields),
                             ctypes.POINTER(ctypes.c_longlong), _VP],
    "gnss_turb_stats": [_VP, ctypes.POINTER(GnssFields), _VP, ctypes.POINTER(ctypes.c_double), _VP],
    "gnss_step_turb": [_VP, ctypes.POINTER(GnssFields), ctypes.POINTER(GnssFields), ctypes.c_int, _VP,
                       ctypes.POINTER(ctypes.c_double), _VP],
    "gnss_attach_scratch": [_VP, _VP, ctypes.c_size_t],
    "gnss_ensemble_create": [ctypes.POINTER(GnssConfig), ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "gnss_ensemble_destroy": [_VP],
    "gnss_ensemble_size": [_VP],
    "gnss_ensemble_member": [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(GnssFields),
                             ctypes.POINTER(GnssFields)],
    "gnss_ensemble_upload": [_VP, ctypes.c_int, _VP, _VP],
    "gnss_ensemble_download": [_VP, ctypes.c_int, _VP, _VP],
    "gnss_ensemble_step": [_VP, ctypes.c_int, _VP],
    "gnss_ensemble_launches_per_step": [_VP],
    "gnss_ensemble_autotune": [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)],
    "gnss_ensemble_set_batching": [_VP, ctypes.c_int],
    "gnss_ensemble_batched": [_VP, ctypes.c_int],
    "gnss_server_create": [_VP, ctypes.POINTER(ctypes.c_void_p)],
    "gnss_server_destroy": [_VP],
    "gnss_server_submit": [_VP, ctypes.POINTER(GnssConfig), _VP, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)],
    "gnss_server_wait": [_VP, ctypes.c_longlong, ctypes.c_double],
    "gnss_server_result": [_VP, ctypes.c_longlong, _VP, ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_double)],
    "gnss_server_report_get": [_VP, _VP],
}
_RESTYPES = {
    "gnss_field_bytes": ctypes.c_size_t,
    "gnss_workspace_bytes": ctypes.c_size_t,
    "gnss_status_string": ctypes.c_char_p,
    "gnss_last_error": ctypes.c_char_p,
    "gnss_launch_count": ctypes.c_longlong,
    "gnss_scratch_bytes": ctypes.c_size_t,
    "gnss_ensemble_size": ctypes.c_int,
    "gnss_ensemble_launches_per_step": ctypes.c_longlong,
}
STAGE_NAMES = ("x_inverse", "y_inverse", "z_physical", "y_forward", "x_forward", "spectral_update")

_lib = None


def load_library(path: Path | str | None = None) -> ctypes.CDLL:
    """Load libgnss_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build the CUDA library first (python gnss-1_b200/build.py)")
    lib = ctypes.CDLL(str(p))
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    if path is None:
        _lib = lib
    return lib


def _ptr(x) -> int | None:
    """Device pointer of a torch tensor (or an int / None passthrough)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    dp = getattr(x, "data_ptr", None)
    if dp is None:
        raise TypeError(f"expected a torch CUDA tensor or a device pointer, got {type(x)!r}")
    if not x.is_cuda:
        raise TypeError("tensor must live on a CUDA device")
    if not x.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return dp()


def _stream(stream) -> int | None:
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except ImportError:
            pass
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _fields(fs: Sequence | None) -> GnssFields | None:
    if fs is None:
        return None
    p = [_ptr(f) for f in fs] + [None] * (5 - len(fs))
    return GnssFields(*p[:5])


def make_config(n: int | None = None, *, nx: int | None = None, ny: int | None = None, nz: int | None = None,
                lx: float = 2 * math.pi, ly: float = 2 * math.pi, lz: float = 2 * math.pi, re: float = 1000.0,
                sc: float = 0.7, sc_c: float = 0.7, alpha: float = 0.0, dt: float = 1e-3,
                alias_filter: float = 2.0 / 3.0, nu_stats: float | None = None, n_scalars: int = 1,
                scheme: int = GNSS_SCHEME_CNAB2, precision: int = GNSS_FP64, device: int = 0) -> GnssConfig:
    """A gnss_config with the reference's defaults (dnsparams.h: LX = LY = LZ = 2 pi, nu = H/Re, H = 1)."""
    nx, ny, nz = nx or n, ny or n, nz or n
    if nu_stats is None:
        nu_stats = 1.0 / re   # the reference's nu = H/Re with H = 1 (dnsparams.h:30)
    return GnssConfig(nx, ny, nz, lx, ly, lz, re, sc, sc_c, alpha, dt, alias_filter, nu_stats,
                      n_scalars, scheme, precision, device)


class Context:
    """One grid configuration on one device (replaces plan1dFFT/plan2dFFT and
    the global state of the reference, fftfuncs.cu:133-231, declare.h)."""

    def __init__(self, n: int | None = None, **kw):
        self.lib = load_library()
        self.cfg = make_config(n, **kw)
        self._owned = True
        h = ctypes.c_void_p()
        st = self.lib.gnss_create(ctypes.byref(self.cfg), ctypes.byref(h))
        if st != GNSS_OK:
            raise GnssError(st, "gnss_create", self.lib.gnss_status_string(st).decode())
        self._h = h

    @classmethod
    def _borrow(cls, handle, cfg: GnssConfig) -> "Context":
        """A view of a context owned elsewhere (an ensemble member); close() does not destroy it."""
        c = cls.__new__(cls)
        c.lib = load_library()
        c.cfg = cfg
        c._owned = False
        c._h = handle
        return c

    # -- bookkeeping -------------------------------------------------------
    @property
    def nz2(self) -> int:
        return self.cfg.nz // 2 + 1

    @property
    def spectral_shape(self) -> tuple:
        return (self.cfg.ny, self.cfg.nx, self.nz2)

    @property
    def complex_dtype(self):
        import torch
        return torch.complex128 if self.cfg.precision == GNSS_FP64 else torch.complex64

    @property
    def n_fields(self) -> int:
        return 3 + self.cfg.n_scalars

    def field_bytes(self) -> int:
        return int(self.lib.gnss_field_bytes(self._h))

    def workspace_bytes(self) -> int:
        return int(self.lib.gnss_workspace_bytes(self._h))

    def empty_field(self, device=None):
        import torch
        return torch.zeros(self.spectral_shape, dtype=self.complex_dtype,
                           device=device if device is not None else f"cuda:{self.cfg.device}")

    def physical_view(self, t):
        """Real padded view [nx, ny, 2*nz2] of a field tensor."""
        import torch
        return torch.view_as_real(t).reshape(self.cfg.nx, self.cfg.ny, 2 * self.nz2)

    def close(self) -> None:
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                self.lib.gnss_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, st: int, what: str) -> None:
        if st != GNSS_OK:
            detail = self.lib.gnss_last_error(self._h)
            raise GnssError(st, what, detail.decode() if detail else "")

    # -- transforms (fftfuncs.cu:288-359) -----------------------------------
    def forward_transform(self, f, stream=None) -> None:
        self._ck(self.lib.gnss_forward(self._h, _ptr(f), _stream(stream)), "gnss_forward")

    def inverse_transform(self, f, stream=None) -> None:
        self._ck(self.lib.gnss_inverse(self._h, _ptr(f), _stream(stream)), "gnss_inverse")

    # -- spectral / physical operators (solver.cu) --------------------------
    def de_alias(self, fields: Iterable, stream=None) -> None:
        for f in fields:
            self._ck(self.lib.gnss_dealias(self._h, _ptr(f), _stream(stream)), "gnss_dealias")

    def vorticity(self, u, v, w, o1, o2, o3, stream=None) -> None:
        self._ck(self.lib.gnss_vorticity(self._h, *map(_ptr, (u, v, w, o1, o2, o3)), _stream(stream)),
                 "gnss_vorticity")

    def gradient(self, f, fx, fy, fz, stream=None) -> None:
        self._ck(self.lib.gnss_gradient(self._h, *map(_ptr, (f, fx, fy, fz)), _stream(stream)), "gnss_gradient")

    def divergence(self, fx, fy, fz, out, stream=None) -> None:
        self._ck(self.lib.gnss_divergence(self._h, *map(_ptr, (fx, fy, fz, out)), _stream(stream)),
                 "gnss_divergence")

    def make_rhs(self, ru, rv, rw, rs=None, rc=None, stream=None) -> None:
        self._ck(self.lib.gnss_make_rhs(self._h, *map(_ptr, (ru, rv, rw, rs, rc)), _stream(stream)),
                 "gnss_make_rhs")

    def timestep(self, euler: bool, state, rhs, rhs_old=None, stream=None) -> None:
        so = _fields(rhs_old)
        self._ck(self.lib.gnss_timestep(self._h, int(bool(euler)), ctypes.byref(_fields(state)),
                                        ctypes.byref(_fields(rhs)), ctypes.byref(so) if so else None,
                                        _stream(stream)), "gnss_timestep")

    def update(self, rhs, rhs_old, stream=None) -> None:
        self._ck(self.lib.gnss_update(self._h, ctypes.byref(_fields(rhs)), ctypes.byref(_fields(rhs_old)),
                                      _stream(stream)), "gnss_update")

    def cross_product(self, u, v, w, o1, o2, o3, stream=None) -> None:
        self._ck(self.lib.gnss_cross_product(self._h, *map(_ptr, (u, v, w, o1, o2, o3)), _stream(stream)),
                 "gnss_cross_product")

    def dot_product(self, a, b, out, stream=None) -> None:
        self._ck(self.lib.gnss_dot_product(self._h, *map(_ptr, (*a, *b, out)), _stream(stream)),
                 "gnss_dot_product")

    def colloid_advection(self, vel, c, grad_c, grad_s, lap_s_inout, stream=None) -> None:
        args = (*vel, c, *grad_c, *grad_s, lap_s_inout)
        self._ck(self.lib.gnss_colloid_advection(self._h, *map(_ptr, args), _stream(stream)),
                 "gnss_colloid_advection")

    # -- the step (solver.cu:700-765) ---------------------------------------
    def solver_ps(self, state: Sequence, hist: Sequence | None, euler: bool, stream=None) -> None:
        h = _fields(hist)
        self._ck(self.lib.gnss_step(self._h, ctypes.byref(_fields(state)), ctypes.byref(h) if h else None,
                                    int(bool(euler)), _stream(stream)), "gnss_step")

    step = solver_ps

    def stats(self, state: Sequence, stream=None) -> dict:
        out = (ctypes.c_double * GNSS_NSTATS)()
        self._ck(self.lib.gnss_stats(self._h, ctypes.byref(_fields(state)), out, _stream(stream)), "gnss_stats")
        return dict(zip(STAT_NAMES, list(out)))

    def run_host(self, host_in, host_out, n_steps: int, first_euler: bool = True, stats=None,
                 stream=None) -> None:
        """End-to-end call: host (ideally pinned) packed state in and out."""
        sp = None
        if stats is not None:
            sp = stats.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if isinstance(stats, np.ndarray) \
                else ctypes.cast(stats.data_ptr(), ctypes.POINTER(ctypes.c_double))
        self._ck(self.lib.gnss_run_host(self._h, _host_ptr(host_in), _host_ptr(host_out), int(n_steps),
                                        int(bool(first_euler)), sp, _stream(stream)), "gnss_run_host")

    def run_host_bytes(self) -> tuple:
        """(host-to-device, device-to-host) state bytes one run_host call copies."""
        h2d, d2h = ctypes.c_size_t(), ctypes.c_size_t()
        self._ck(self.lib.gnss_run_host_bytes(self._h, ctypes.byref(h2d), ctypes.byref(d2h)), "gnss_run_host_bytes")
        return h2d.value, d2h.value

    def check(self, stream=None) -> None:
        """Synchronise and raise if a bounded device wait timed out."""
        self._ck(self.lib.gnss_check(self._h, _stream(stream)), "gnss_check")

    # -- instrumentation ------------------------------------------------------
    def launch_count(self) -> int:
        return int(self.lib.gnss_launch_count(self._h))

    def turb_stats(self, state: Sequence, profiles: bool = True, stream=None):
        """calcTurbStats_mgpu (statistics.cu:2039-2156): (dict, mean y-profiles [5, ny] of u, v, w, s, c)."""
        t = GnssTurb()
        prof = np.zeros((5, self.cfg.ny)) if profiles else None
        pp = prof.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if prof is not None else None
        f = _fields(state)
        self._ck(self.lib.gnss_turb_stats(self._h, ctypes.byref(f), ctypes.byref(t), pp, _stream(stream)),
                 "gnss_turb_stats")
        d = {k: getattr(t, k) for k, _ in GnssTurb._fields_}
        d["lambda"] = d.pop("lambda_")
        return d, prof

    def step_turb(self, state: Sequence, hist: Sequence | None, euler: bool, profiles: bool = True, stream=None):
        """One step plus turb_stats of the state it starts from; the vorticity statistics are summed by the
        step's own z kernel where the register kernel serves the context."""
        t = GnssTurb()
        prof = np.zeros((5, self.cfg.ny)) if profiles else None
        pp = prof.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if prof is not None else None
        h = _fields(hist)
        self._ck(self.lib.gnss_step_turb(self._h, ctypes.byref(_fields(state)), ctypes.byref(h) if h else None,
                                         int(bool(euler)), ctypes.byref(t), pp, _stream(stream)), "gnss_step_turb")
        d = {k: getattr(t, k) for k, _ in GnssTurb._fields_}
        d["lambda"] = d.pop("lambda_")
        return d, prof

    def initial_jet(self, state: Sequence, h: float = 1.0, theta: float = 0.05, theta_c: float = 0.05,
                    pert_amp: float = 0.05, seed: int = 0, stream=None) -> None:
        """The reference's initializeJet (initialize.cu:615-641) + forward transforms + dealias (main.cu:149-156)."""
        p = GnssJetParams(h, theta, theta_c, pert_amp, seed)
        f = _fields(state)
        self._ck(self.lib.gnss_initial_jet(self._h, ctypes.byref(p), ctypes.byref(f), _stream(stream)),
                 "gnss_initial_jet")

    # -- files (iofuncs.cu formats, exact checkpoint) -------------------------
    def save_state(self, state: Sequence, directory, iteration: int, stream=None) -> None:
        """save3Dfields (iofuncs.cu:360-432): <dir>/u.<iter>, v, w, z, c in physical space."""
        f = _fields(state)
        self._ck(self.lib.gnss_save_state(self._h, ctypes.byref(f), str(directory).encode(), int(iteration),
                                          _stream(stream)), "gnss_save_state")

    def load_state(self, directory, iteration: int, state: Sequence, stream=None) -> None:
        """importVelocity / importScalar + forward transforms into `state`."""
        f = _fields(state)
        self._ck(self.lib.gnss_load_state(self._h, str(directory).encode(), int(iteration), ctypes.byref(f),
                                          _stream(stream)), "gnss_load_state")

    def checkpoint_save(self, state: Sequence, hist: Sequence | None, step: int, path, stream=None) -> None:
        f, h = _fields(state), _fields(hist)
        self._ck(self.lib.gnss_checkpoint_save(self._h, ctypes.byref(f), ctypes.byref(h) if h else None, int(step),
                                               str(path).encode(), _stream(stream)), "gnss_checkpoint_save")

    def checkpoint_load(self, path, state: Sequence, hist: Sequence | None, stream=None) -> int:
        f, h = _fields(state), _fields(hist)
        step = ctypes.c_longlong()
        self._ck(self.lib.gnss_checkpoint_load(self._h, str(path).encode(), ctypes.byref(f),
                                               ctypes.byref(h) if h else None, ctypes.byref(step), _stream(stream)),
                 "gnss_checkpoint_load")
        return step.value

    def set_option(self, key: int, value: int) -> None:
        self._ck(self.lib.gnss_set_option(self._h, key, value), "gnss_set_option")

    def get_option(self, key: int) -> int:
        v = ctypes.c_int()
        self._ck(self.lib.gnss_get_option(self._h, key, ctypes.byref(v)), "gnss_get_option")
        return v.value

    def stage_bytes(self) -> dict:
        """Algorithmic HBM bytes of one launch of each stage of the step."""
        b = (ctypes.c_double * len(STAGE_NAMES))()
        self._ck(self.lib.gnss_stage_bytes(self._h, b), "gnss_stage_bytes")
        return {k: float(b[i]) for i, k in enumerate(STAGE_NAMES)}

    def profile(self, on: bool) -> None:
        self._ck(self.lib.gnss_profile_enable(self._h, int(bool(on))), "gnss_profile_enable")

    def profile_read(self) -> dict:
        ms = (ctypes.c_double * len(STAGE_NAMES))()
        n = (ctypes.c_longlong * len(STAGE_NAMES))()
        self._ck(self.lib.gnss_profile_read(self._h, ms, n), "gnss_profile_read")
        return {k: (ms[i], int(n[i])) for i, k in enumerate(STAGE_NAMES)}

    # reference spellings
    forwardTransform = forward_transform
    inverseTransform = inverse_transform
    deAlias = de_alias
    makeRHS = make_rhs
    crossProduct = cross_product
    dotProduct = dot_product
    colloidAdvection = colloid_advection


def _host_ptr(x) -> int:
    if isinstance(x, np.ndarray):
        assert x.flags.c_contiguous
        return x.ctypes.data
    if isinstance(x, int):
        return x
    if x.is_cuda:
        raise TypeError("run_host expects host memory")
    return x.data_ptr()


# ---------------------------------------------------------------- initial state
def _splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
    z = x
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _normals(seed: int, keys: np.ndarray) -> np.ndarray:
    """Counter-based standard normals: one per uint64 key, reproducible on any machine."""
    with np.errstate(over="ignore"):
        s = _splitmix64(np.array([seed], dtype=np.uint64))[0]
        k2 = keys.astype(np.uint64) * np.uint64(2)
        a = _splitmix64(k2 ^ s)
        b = _splitmix64((k2 + np.uint64(1)) ^ s)
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
    u2 = ((b >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def jet_profile(ny: int, ly: float, h: float = 1.0, theta: float = 0.05) -> np.ndarray:
    """Temporal-jet profile on the y grid (initialize.cu:114-136, 161-177):
    0.5 - 0.5 tanh(H/(4 theta) (2|y|/H - 1)) with y = -ly/2 + j ly/ny."""
    y = -ly / 2 + np.arange(ny) * ly / ny
    return 0.5 - 0.5 * np.tanh(h / (4.0 * theta) * (2.0 * np.abs(y) / h - 1.0))


def jet_initial_state(nx: int, ny: int | None = None, nz: int | None = None, *, lx: float = 2 * math.pi,
                      ly: float = 2 * math.pi, lz: float = 2 * math.pi, n_scalars: int = 1, seed: int = 0,
                      noise_kmax: float = 8.0, amp: float = 0.05, h: float = 1.0, theta: float = 0.05,
                      dtype=np.complex128) -> list:
    """Seeded spectral initial state [u, v, w, s(, c)], each complex [ny][nx][nz2].

    u = U(y) + noise, v, w = noise, s (and c) = U(y).  The noise is the
    solenoidal field i k x A on the modes 0 < |k| <= noise_kmax with A drawn
    from a counter-based generator keyed by ``seed``, Hermitian in the kz = 0
    plane, scaled so that the mean component rms in physical space is ``amp``.
    """
    ny = ny or nx
    nz = nz or nx
    nz2 = nz // 2 + 1
    nn = float(nx) * ny * nz
    dkx, dky, dkz = 2 * math.pi / lx, 2 * math.pi / ly, 2 * math.pi / lz
    fields = [np.zeros((ny, nx, nz2), dtype=dtype) for _ in range(3 + n_scalars)]
    prof = np.fft.fft(jet_profile(ny, ly, h, theta)) * (nx * nz)
    fields[0][:, 0, 0] = prof
    for q in range(3, 3 + n_scalars):
        fields[q][:, 0, 0] = prof
    if amp > 0 and noise_kmax > 0:
        kx_n = int(math.floor(noise_kmax / dkx))
        ky_n = int(math.floor(noise_kmax / dky))
        kz_n = int(math.floor(noise_kmax / dkz))
        kx_n = min(kx_n, nx // 2 - 1)
        ky_n = min(ky_n, ny // 2 - 1)
        kz_n = min(kz_n, nz // 2 - 1)
        mx, my, mz = np.meshgrid(np.arange(-kx_n, kx_n + 1), np.arange(-ky_n, ky_n + 1), np.arange(0, kz_n + 1),
                                 indexing="ij")
        mx, my, mz = mx.ravel(), my.ravel(), mz.ravel()
        kx, ky, kz = mx * dkx, my * dky, mz * dkz
        k2 = kx * kx + ky * ky + kz * kz
        canon = (mz > 0) | ((mz == 0) & ((my > 0) | ((my == 0) & (mx > 0))))
        sel = (k2 > 0) & (k2 <= noise_kmax ** 2 * (1 + 1e-12)) & canon
        mx, my, mz, kx, ky, kz = mx[sel], my[sel], mz[sel], kx[sel], ky[sel], kz[sel]
        base = ((mx + 1024).astype(np.int64) * 2048 + (my + 1024)) * 2048 + mz
        a = np.empty((3, mx.size), dtype=np.complex128)
        for comp in range(3):
            re_ = _normals(seed, base * 8 + 2 * comp)
            im_ = _normals(seed, base * 8 + 2 * comp + 1)
            a[comp] = (re_ + 1j * im_) / math.sqrt(2.0)
        kv = np.stack([kx, ky, kz])
        # n = i k x A
        cross = np.stack([ky * a[2] - kz * a[1], kz * a[0] - kx * a[2], kx * a[1] - ky * a[0]])
        nh = 1j * cross
        wt = np.where(mz > 0, 2.0, 1.0)
        # mirrored kz = 0 modes contribute once more
        wt = np.where(mz == 0, 2.0, wt)
        var = (wt * np.abs(nh) ** 2).sum(axis=1) / nn ** 2
        scale = amp / math.sqrt(var.mean()) if var.mean() > 0 else 0.0
        nh *= scale
        iy, ix = my % ny, mx % nx
        for comp in range(3):
            fields[comp][iy, ix, mz] += nh[comp].astype(dtype)
            z0 = mz == 0
            fields[comp][(-my[z0]) % ny, (-mx[z0]) % nx, 0] += np.conj(nh[comp][z0]).astype(dtype)
        del kv
    return fields


def pack_state(fields: Sequence[np.ndarray], out: np.ndarray | None = None) -> np.ndarray:
    """Back-to-back copy of fields (the layout gnss_run_host expects)."""
    n = fields[0].size
    if out is None:
        out = np.empty(n * len(fields), dtype=fields[0].dtype)
    for q, f in enumerate(fields):
        out[q * n:(q + 1) * n] = f.ravel()
    return out


# ---------------------------------------------------------------------- batching
class Ensemble:
    """Many independent jets stepped together (gnss_ensemble_*): every member's
    steps after the first are one CUDA graph launch.  configs: GnssConfig
    values (make_config); all on one device."""

    def __init__(self, configs: Sequence[GnssConfig], n_branches: int = 4):
        self.lib = load_library()
        self.configs = list(configs)
        arr = (GnssConfig * len(self.configs))(*self.configs)
        h = ctypes.c_void_p()
        st = self.lib.gnss_ensemble_create(arr, len(self.configs), int(n_branches), ctypes.byref(h))
        if st != GNSS_OK:
            raise GnssError(st, "gnss_ensemble_create", self.lib.gnss_status_string(st).decode())
        self._h = h

    def __len__(self) -> int:
        return int(self.lib.gnss_ensemble_size(self._h))

    def member(self, i: int):
        """(Context view, state GnssFields, history GnssFields) of member i."""
        ch = ctypes.c_void_p()
        sf, hf = GnssFields(), GnssFields()
        self._ck(self.lib.gnss_ensemble_member(self._h, i, ctypes.byref(ch), ctypes.byref(sf), ctypes.byref(hf)),
                 "gnss_ensemble_member")
        return Context._borrow(ch, self.configs[i]), sf, hf

    def upload(self, i: int, host_state, stream=None) -> None:
        self._ck(self.lib.gnss_ensemble_upload(self._h, i, _host_ptr(host_state), _stream(stream)),
                 "gnss_ensemble_upload")

    def download(self, i: int, host_state, stream=None) -> None:
        self._ck(self.lib.gnss_ensemble_download(self._h, i, _host_ptr(host_state), _stream(stream)),
                 "gnss_ensemble_download")

    def step(self, n_steps: int, stream=None) -> None:
        self._ck(self.lib.gnss_ensemble_step(self._h, int(n_steps), _stream(stream)), "gnss_ensemble_step")

    def launches_per_step(self) -> int:
        return int(self.lib.gnss_ensemble_launches_per_step(self._h))

    def set_batching(self, on: bool) -> None:
        """Groups of one geometry step as one batched launch per stage (on) or member by member."""
        self._ck(self.lib.gnss_ensemble_set_batching(self._h, 1 if on else 0), "gnss_ensemble_set_batching")

    def batched(self, i: int) -> bool:
        """Whether member i's group steps as batched launches."""
        return int(self.lib.gnss_ensemble_batched(self._h, int(i))) == 1

    def autotune(self, steps: int = 3) -> list:
        ch = (ctypes.c_int * len(self.configs))()
        self._ck(self.lib.gnss_ensemble_autotune(self._h, int(steps), ch), "gnss_ensemble_autotune")
        return list(ch)

    def stats(self, i: int, stream=None) -> dict:
        ctx, sf, _ = self.member(i)
        out = (ctypes.c_double * GNSS_NSTATS)()
        self._ck(self.lib.gnss_stats(ctx._h, ctypes.byref(sf), out, _stream(stream)), "gnss_stats")
        return {k: float(out[j]) for j, k in enumerate(STAT_NAMES)}

    def points(self) -> float:
        return float(sum(c.nx * c.ny * c.nz for c in self.configs))

    def _ck(self, st: int, what: str) -> None:
        if st != GNSS_OK:
            raise GnssError(st, what, self.lib.gnss_status_string(st).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.gnss_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class ServerConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_size_t), ("max_active", ctypes.c_int),
                ("steps_per_launch", ctypes.c_int), ("device", ctypes.c_int)]


class ServerReport(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("admitted", ctypes.c_longlong),
                ("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("bytes_reserved", ctypes.c_size_t), ("bytes_reserved_max", ctypes.c_size_t),
                ("active_max", ctypes.c_int), ("point_steps", ctypes.c_double),
                ("busy_seconds", ctypes.c_double)]


class Server:
    """Continuous-batching request loop (gnss_server_*): jets are admitted in
    arrival order under a device-memory budget, stay resident while they run,
    and advance concurrently on their own streams."""

    def __init__(self, budget_bytes: int, max_active: int = 32, steps_per_launch: int = 20, device: int = 0):
        self.lib = load_library()
        cfg = ServerConfig(int(budget_bytes), int(max_active), int(steps_per_launch), int(device))
        h = ctypes.c_void_p()
        st = self.lib.gnss_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != GNSS_OK:
            raise GnssError(st, "gnss_server_create", self.lib.gnss_status_string(st).decode())
        self._h = h
        self._shapes = {}

    def submit(self, cfg: GnssConfig, host_state: np.ndarray, n_steps: int) -> int:
        """Queue a jet run; host_state: packed fields (pack_state), copied at submission."""
        a = np.ascontiguousarray(host_state)
        rid = ctypes.c_longlong()
        st = self.lib.gnss_server_submit(self._h, ctypes.byref(cfg), a.ctypes.data, int(n_steps), ctypes.byref(rid))
        if st != GNSS_OK:
            raise GnssError(st, "gnss_server_submit", self.lib.gnss_status_string(st).decode())
        self._shapes[rid.value] = (a.shape, a.dtype)
        return rid.value

    def wait(self, rid: int, timeout: float = 600.0) -> None:
        st = self.lib.gnss_server_wait(self._h, int(rid), float(timeout))
        if st != GNSS_OK:
            raise GnssError(st, "gnss_server_wait", self.lib.gnss_status_string(st).decode())

    def result(self, rid: int):
        """(final packed state, statistics dict, (submitted, admitted, finished) seconds)."""
        shape, dtype = self._shapes.pop(rid)
        out = np.empty(shape, dtype=dtype)
        stats = (ctypes.c_double * GNSS_NSTATS)()
        times = (ctypes.c_double * 3)()
        st = self.lib.gnss_server_result(self._h, int(rid), out.ctypes.data, stats, times)
        if st != GNSS_OK:
            raise GnssError(st, "gnss_server_result", self.lib.gnss_status_string(st).decode())
        return out, {k: float(stats[j]) for j, k in enumerate(STAT_NAMES)}, tuple(times)

    def report(self) -> dict:
        r = ServerReport()
        st = self.lib.gnss_server_report_get(self._h, ctypes.byref(r))
        if st != GNSS_OK:
            raise GnssError(st, "gnss_server_report_get")
        return {k: getattr(r, k) for k, _ in ServerReport._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.gnss_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ---------------------------------------------------------------------- reference file formats
GNSS_PLANE_XY, GNSS_PLANE_XZ, GNSS_PLANE_YZ = 0, 1, 2


def _io_ck(st: int, what: str) -> None:
    if st != GNSS_OK:
        raise GnssError(st, what)


def padded_shape(nx: int, ny: int, nz: int) -> tuple:
    """Shape of a physical field in the reference's in-place layout."""
    return (nx, ny, 2 * (nz // 2 + 1))


def io_write_field(phys: np.ndarray, nz: int, path) -> None:
    """write3Dfields_mgpu (iofuncs.cu:329-358): phys float64 [nx][ny][2 nz2]."""
    a = np.ascontiguousarray(phys, dtype=np.float64)
    _io_ck(load_library().gnss_io_write_field(a.shape[0], a.shape[1], nz, a.ctypes.data, str(path).encode()),
           "gnss_io_write_field")


def io_read_field(nx: int, ny: int, nz: int, path) -> np.ndarray:
    """loadData (iofuncs.cu:462-497) into a zero-padded array [nx][ny][2 nz2]."""
    a = np.zeros(padded_shape(nx, ny, nz))
    _io_ck(load_library().gnss_io_read_field(nx, ny, nz, str(path).encode(), a.ctypes.data), "gnss_io_read_field")
    return a


def io_write_slice(phys: np.ndarray, nz: int, plane: int, index: int, path) -> None:
    a = np.ascontiguousarray(phys, dtype=np.float64)
    _io_ck(load_library().gnss_io_write_slice(a.shape[0], a.shape[1], nz, a.ctypes.data, int(plane), int(index),
                                              str(path).encode()), "gnss_io_write_slice")


def io_write_stat(path, value: float, append: bool) -> None:
    _io_ck(load_library().gnss_io_write_stat(str(path).encode(), float(value), int(bool(append))),
           "gnss_io_write_stat")


def io_write_profile(prof: np.ndarray, path) -> None:
    a = np.ascontiguousarray(prof, dtype=np.float64)
    _io_ck(load_library().gnss_io_write_profile(a.size, a.ctypes.data, str(path).encode()), "gnss_io_write_profile")
