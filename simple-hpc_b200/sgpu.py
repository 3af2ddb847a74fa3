"""Python binding of the B200 SIMPLE solver's C ABI (include/sgpu.h), via ctypes.

`Solver` mirrors the reference's GPU backend class `HipSolver` (include/simple/solver_hip.hpp:11-37):
one method per phase (assemble_u, bc_u, residual_u, sweep_u, ... correct), `outer_iteration`,
`download`, and `run` for the outer loop with the reference's stopping rule (run_outer_loop,
src/solver.cpp:106-132). Errors come back as `SgpuError` carrying the library's message, the way
HipSolver throws std::runtime_error("GPU error: ...").

There is no CPU fallback: if libsgpu.so is missing or cannot be loaded, importing the library raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("SGPU_LIB", HERE / "libsgpu.so"))

SGPU_OK = 0
E_INVALID, E_CUDA, E_NOMEM, E_TIMEOUT, E_NONFINITE, E_NODEVICE = -1, -2, -3, -4, -5, -6

UDS, QUICK = 0, 1
NORM_ABSOLUTE, NORM_RUNNING_MAX = 0, 1
MOM_GS_LEX, MOM_JACOBI, MOM_GS_MULTICOLOUR = 0, 1, 2
P_GS_LEX, P_JACOBI, P_GS_REDBLACK, P_CG, P_MG = 0, 1, 2, 3, 4
PREC_FP64, PREC_MIXED = 0, 1

# Field ids (include/sgpu.h).
F_U, F_V, F_P = 0, 1, 2
CU = list(range(3, 12))   # AE AW AN AS AEE AWW ANN ASS AP of u
CV = list(range(12, 21))
F_AEP, F_AWP, F_ANP, F_ASP, F_APP, F_B, F_PC = range(21, 28)
FIELD_COUNT = 28
COEF_NAMES = ["AE", "AW", "AN", "AS", "AEE", "AWW", "ANN", "ASS", "AP"]
FIELD_NAMES = (["u", "v", "p"] + [f"cu.{n}" for n in COEF_NAMES] + [f"cv.{n}" for n in COEF_NAMES]
               + ["AEP", "AWP", "ANP", "ASP", "APP", "b", "pc"])
PHASES = ["assemble_u", "bc_u", "residual_u", "sweep_u", "assemble_v", "bc_v", "residual_v",
          "sweep_v", "assemble_p", "solve_p", "correct", "output"]


class Params(C.Structure):
    """sgpu_params_t: the reference's struct Params (include/simple/params.hpp:15-58) as plain data."""

    _fields_ = [
        ("NX", C.c_int), ("NY", C.c_int), ("H", C.c_int), ("N_halo_x", C.c_int), ("N_halo_y", C.c_int),
        ("Re", C.c_double),
        ("maxit_inner_u", C.c_int), ("maxit_inner_v", C.c_int), ("maxit_inner_p", C.c_int),
        ("error_tolerance", C.c_double), ("maxit", C.c_int),
        ("relaxation_factor_u", C.c_double), ("relaxation_factor_v", C.c_double),
        ("relaxation_factor_p", C.c_double),
        ("convection_scheme", C.c_int), ("diffusion_order", C.c_int), ("hybrid_switch", C.c_int),
        ("residual_normalisation", C.c_int), ("backend", C.c_int), ("momentum_solver", C.c_int),
        ("pressure_solver", C.c_int), ("pressure_tolerance", C.c_double), ("pressure_maxit", C.c_int),
        ("mg_cycles", C.c_int), ("mg_pre", C.c_int), ("mg_post", C.c_int), ("mg_omega", C.c_double),
        ("halo_overlap", C.c_int), ("write_fields", C.c_int),
        ("grid_rows_cfg", C.c_int), ("grid_cols_cfg", C.c_int),
        ("precision", C.c_int), ("mg_mode", C.c_int), ("warm_start", C.c_int), ("graph_batch", C.c_int),
        ("nrows", C.c_int), ("ncols", C.c_int), ("dx", C.c_double), ("dy", C.c_double), ("nu", C.c_double),
        ("output_dir", C.c_char * 512), ("cnn_weights", C.c_char * 512),
        ("restart_from", C.c_char * 512),
    ]

    @property
    def shape(self) -> tuple[int, int]:
        return (self.nrows, self.ncols)


class Result(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("seconds", C.c_double),
                ("phase_seconds", C.c_double * 12), ("cg_iterations", C.c_longlong),
                ("mg_vcycles", C.c_longlong)]


class SgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load libsgpu.so (fails loudly: the solver has no CPU path)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with simple-hpc_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        P, D, I, H = C.POINTER(Params), C.POINTER(C.c_double), C.c_int, C.c_void_p
        F = C.POINTER(C.c_float)
        sig = {
            "sgpu_params_from_config": (I, [C.c_char_p, P]),
            "sgpu_params_default": (I, [P]),
            "sgpu_params_finalize": (I, [P]),
            "sgpu_last_error": (C.c_char_p, []),
            "sgpu_version": (C.c_char_p, []),
            "sgpu_create": (I, [P, D, D, D, C.POINTER(H)]),
            "sgpu_destroy": (I, [H]),
            "sgpu_assemble_u": (I, [H]), "sgpu_bc_u": (I, [H]), "sgpu_residual_u": (I, [H, D]),
            "sgpu_sweep_u": (I, [H, I]), "sgpu_assemble_v": (I, [H]), "sgpu_bc_v": (I, [H]),
            "sgpu_residual_v": (I, [H, D]), "sgpu_sweep_v": (I, [H, I]),
            "sgpu_assemble_p": (I, [H, D]), "sgpu_solve_p": (I, [H]), "sgpu_correct": (I, [H]),
            "sgpu_outer_iteration": (I, [H, D, D]),
            "sgpu_run": (I, [H, I, D, I, C.POINTER(Result)]),
            "sgpu_download": (I, [H, I, D]), "sgpu_upload": (I, [H, I, D]),
            "sgpu_memory_bytes": (I, [H, C.POINTER(C.c_size_t)]),
            "sgpu_selftest_bounded_wait": (I, [I, C.POINTER(I)]),
            "sgpu_mg_levels": (I, [I, I, C.POINTER(I), C.POINTER(I)]),
            "sgpu_last_solve_stats": (I, [H, C.POINTER(I), C.POINTER(I), C.POINTER(I), D]),
            "sgpu_ordered_sum": (I, [D, I, I, D]),
            "sgpu_set_profiling": (I, [H, I]), "sgpu_phase_seconds": (I, [H, D]),
            "sgpu_sweep_seconds": (I, [H, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
            "sgpu_stream": (I, [H, C.POINTER(C.c_void_p)]), "sgpu_launch_count": (C.c_longlong, []),
            "sgpu_write_outputs": (I, [P, D, D, D, D, I, C.POINTER(Result), C.c_char_p, C.c_char_p,
                                       C.c_char_p]),
            "sgpu_read_fields": (I, [P, C.c_char_p, D, D, D]),
            # learned warm start
            "sgpu_cnn_load": (I, [H, C.c_char_p]),
            "sgpu_cnn_create": (I, [I, I, C.c_uint, C.POINTER(H)]),
            "sgpu_cnn_read": (I, [C.c_char_p, C.POINTER(H)]),
            "sgpu_cnn_write": (I, [H, C.c_char_p]),
            "sgpu_cnn_destroy": (I, [H]),
            "sgpu_cnn_info": (I, [H, C.POINTER(I), C.POINTER(I), C.POINTER(C.c_longlong), D]),
            "sgpu_cnn_get_params": (I, [H, F]), "sgpu_cnn_set_params": (I, [H, F]),
            "sgpu_cnn_forward": (I, [H, F, I, I, I, F]),
            "sgpu_cnn_loss_grad": (I, [H, F, F, I, I, I, F, F]),
            "sgpu_cnn_train_step": (I, [H, F, F, I, I, I, C.c_float, F]),
            "sgpu_attach_cnn": (I, [H, H, I]),
            "sgpu_warm_start_stats": (I, [H, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), D]),
            "sgpu_set_mg_mode": (I, [H, I, C.c_double, I]),
            "sgpu_cnn_sample": (I, [H, I, F, F, C.POINTER(I), C.POINTER(I), C.POINTER(I)]),
            # batched cavities
            "sgpu_batch_create": (I, [P, I, C.POINTER(H)]),
            "sgpu_batch_destroy": (I, [H]),
            "sgpu_batch_count": (I, [H, C.POINTER(I)]),
            "sgpu_batch_autotune": (I, [H, C.POINTER(I)]),
            "sgpu_batch_run": (I, [H, I, I, D]),
            "sgpu_batch_results": (I, [H, C.POINTER(I), C.POINTER(I), D]),
            "sgpu_batch_log": (I, [H, D]),
            "sgpu_batch_download": (I, [H, I, I, D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != SGPU_OK:
        raise SgpuError(rc, lib().sgpu_last_error().decode())


def _dptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Batch:
    """Independent cavities solved in one graph launch (sgpu_batch_*)."""

    def __init__(self, params: list[Params]):
        arr = (Params * len(params))(*params)
        h = C.c_void_p()
        _check(lib().sgpu_batch_create(arr, len(params), C.byref(h)))
        self._h = h
        self.params = list(params)
        self.log_cap = 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().sgpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def autotune(self) -> list[int]:
        out = (C.c_int * len(self.params))()
        _check(lib().sgpu_batch_autotune(self._h, out))
        return list(out)

    def run(self, maxit: int, log_cap: int = 0) -> float:
        """Run all cavities; returns the device seconds of the launch."""
        sec = C.c_double()
        _check(lib().sgpu_batch_run(self._h, maxit, log_cap, C.byref(sec)))
        self.log_cap = log_cap
        return sec.value

    def results(self) -> dict:
        n = len(self.params)
        its, conv = (C.c_int * n)(), (C.c_int * n)()
        res = np.zeros((n, 3))
        _check(lib().sgpu_batch_results(self._h, its, conv, _dptr(res)))
        conv = np.array(conv)
        return {"iterations": np.array(its), "converged": conv == 1, "diverged": conv == -1,
                "residuals": res}

    def log(self) -> np.ndarray:
        out = np.zeros((len(self.params), self.log_cap, 4))
        _check(lib().sgpu_batch_log(self._h, _dptr(out)))
        return out

    def download(self, index: int, field_id: int) -> np.ndarray:
        p = self.params[index]
        out = np.empty((p.nrows, p.ncols))
        _check(lib().sgpu_batch_download(self._h, index, field_id, _dptr(out)))
        return out


class Cnn:
    """The warm-start network (sgpu_cnn_*): U-Net with BF16 tensor-core kernels, trained on the GPU.

    Images are (n, height, width, 2) FP32 inputs and (n, height, width) FP32 targets / outputs;
    height and width must be multiples of 2^(levels - 1)."""

    def __init__(self, base: int = 16, levels: int = 4, seed: int = 0, path: str | None = None):
        h = C.c_void_p()
        if path is not None:
            _check(lib().sgpu_cnn_read(str(path).encode(), C.byref(h)))
        else:
            _check(lib().sgpu_cnn_create(base, levels, seed, C.byref(h)))
        self._h = h
        b, l, n, f = C.c_int(), C.c_int(), C.c_longlong(), C.c_double()
        _check(lib().sgpu_cnn_info(h, C.byref(b), C.byref(l), C.byref(n), C.byref(f)))
        self.base, self.levels, self.num_params, self.flops_per_pixel = b.value, l.value, n.value, f.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().sgpu_cnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def write(self, path) -> None:
        _check(lib().sgpu_cnn_write(self._h, str(path).encode()))

    def params(self) -> np.ndarray:
        out = np.empty(self.num_params, np.float32)
        _check(lib().sgpu_cnn_get_params(self._h, _fptr(out)))
        return out

    def set_params(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32)
        if w.shape != (self.num_params,):
            raise ValueError(f"expected {self.num_params} parameters, got {w.shape}")
        _check(lib().sgpu_cnn_set_params(self._h, _fptr(w)))

    @staticmethod
    def _images(x: np.ndarray) -> tuple[np.ndarray, int, int, int]:
        x = np.ascontiguousarray(x, np.float32)
        if x.ndim != 4 or x.shape[3] != 2:
            raise ValueError(f"input must be (n, height, width, 2), got {x.shape}")
        return x, x.shape[0], x.shape[1], x.shape[2]

    def forward(self, x: np.ndarray) -> np.ndarray:
        x, n, hh, ww = self._images(x)
        out = np.empty((n, hh, ww), np.float32)
        _check(lib().sgpu_cnn_forward(self._h, _fptr(x), n, hh, ww, _fptr(out)))
        return out

    def loss_grad(self, x: np.ndarray, t: np.ndarray) -> tuple[float, np.ndarray]:
        x, n, hh, ww = self._images(x)
        t = np.ascontiguousarray(t, np.float32).reshape(n, hh, ww)
        g = np.empty(self.num_params, np.float32)
        loss = C.c_float()
        _check(lib().sgpu_cnn_loss_grad(self._h, _fptr(x), _fptr(t), n, hh, ww, C.byref(loss), _fptr(g)))
        return loss.value, g

    def train_step(self, x: np.ndarray, t: np.ndarray, lr: float) -> float:
        x, n, hh, ww = self._images(x)
        t = np.ascontiguousarray(t, np.float32).reshape(n, hh, ww)
        loss = C.c_float()
        _check(lib().sgpu_cnn_train_step(self._h, _fptr(x), _fptr(t), n, hh, ww, lr, C.byref(loss)))
        return loss.value


def params_from_config(text: str, **overrides) -> Params:
    """make_params(parse_config(text)) with optional key = value overrides appended as text."""
    if overrides:
        lines = [ln for ln in text.splitlines()
                 if ln.split("#")[0].split("=")[0].strip() not in overrides]
        text = "\n".join(lines + [f"{k} = {v}" for k, v in overrides.items()])
    p = Params()
    _check(lib().sgpu_params_from_config(text.encode(), C.byref(p)))
    return p


def params_from_file(path: str | os.PathLike, **overrides) -> Params:
    return params_from_config(Path(path).read_text(), **overrides)


def mg_levels(nx: int, ny: int) -> list[tuple[int, int]]:
    n = C.c_int()
    dims = (C.c_int * 128)()
    _check(lib().sgpu_mg_levels(nx, ny, C.byref(n), dims))
    return [(dims[2 * k], dims[2 * k + 1]) for k in range(n.value)]


def write_outputs(p: Params, u: np.ndarray, v: np.ndarray, pf: np.ndarray, log: np.ndarray,
                  result: Result | None = None, cfg_path: str = "", git_hash: str = "unknown",
                  compiler: str = "unknown") -> None:
    """The reference's output files from host arrays (write_outputs, src/io.cpp:43-151)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, pf)]
    lg = np.ascontiguousarray(log, dtype=np.float64).reshape(-1, 4)
    if result is None:
        result = Result()
        result.iterations = lg.shape[0]
    _check(lib().sgpu_write_outputs(C.byref(p), *(_dptr(a) for a in arrs), _dptr(lg), lg.shape[0],
                                    C.byref(result), cfg_path.encode(), git_hash.encode(),
                                    compiler.encode()))


def read_fields(p: Params, directory) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """u, v, p from the u.csv, v.csv, p.csv a run wrote into `directory` (restart_from)."""
    out = [np.empty((p.nrows, p.ncols)) for _ in range(3)]
    _check(lib().sgpu_read_fields(C.byref(p), str(directory).encode(), *(_dptr(a) for a in out)))
    return out[0], out[1], out[2]


def launch_count() -> int:
    return int(lib().sgpu_launch_count())


def selftest_bounded_wait(polls: int = 4096) -> bool:
    """Run the device-side failure-detection diagnostic (sgpu_selftest_bounded_wait): True when a
    bounded wait on an mbarrier that never completes gave up and reported it."""
    out = C.c_int(0)
    _check(lib().sgpu_selftest_bounded_wait(int(polls), C.byref(out)))
    return bool(out.value)


def ordered_sum(values: np.ndarray) -> float:
    v = np.ascontiguousarray(values, dtype=np.float64)
    if v.ndim == 1:
        v = v.reshape(1, -1)
    out = C.c_double()
    _check(lib().sgpu_ordered_sum(_dptr(v), v.shape[0], v.shape[1], C.byref(out)))
    return out.value


class Solver:
    """One solver on the current CUDA device: the reference's HipSolver (solver_hip.hpp:11-37)."""

    def __init__(self, p: Params, u: np.ndarray | None = None, v: np.ndarray | None = None,
                 pf: np.ndarray | None = None):
        self.p = p
        self.shape = (p.nrows, p.ncols)
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, pf)]
        for a in arrs:
            if a is not None and a.shape != self.shape:
                raise ValueError(f"field shape {a.shape} != {self.shape}")
        h = C.c_void_p()
        _check(lib().sgpu_create(C.byref(p), *(_dptr(a) for a in arrs), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().sgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # per-phase entry points (HipSolver members)
    def assemble_u(self): _check(lib().sgpu_assemble_u(self._h))
    def bc_u(self): _check(lib().sgpu_bc_u(self._h))
    def sweep_u(self, n: int): _check(lib().sgpu_sweep_u(self._h, n))
    def assemble_v(self): _check(lib().sgpu_assemble_v(self._h))
    def bc_v(self): _check(lib().sgpu_bc_v(self._h))
    def sweep_v(self, n: int): _check(lib().sgpu_sweep_v(self._h, n))
    def solve_p(self): _check(lib().sgpu_solve_p(self._h))
    def correct(self): _check(lib().sgpu_correct(self._h))

    def residual_u(self) -> float:
        r = C.c_double()
        _check(lib().sgpu_residual_u(self._h, C.byref(r)))
        return r.value

    def residual_v(self) -> float:
        r = C.c_double()
        _check(lib().sgpu_residual_v(self._h, C.byref(r)))
        return r.value

    def assemble_p(self) -> float:
        r = C.c_double()
        _check(lib().sgpu_assemble_p(self._h, C.byref(r)))
        return r.value

    def outer_iteration(self, phase_seconds: np.ndarray | None = None) -> tuple[float, float, float]:
        res = np.zeros(3)
        _check(lib().sgpu_outer_iteration(self._h, _dptr(res), _dptr(phase_seconds)))
        return float(res[0]), float(res[1]), float(res[2])

    def run(self, maxit: int | None = None, print_every: int = 0):
        """Outer loop; returns (Result, log[iterations, 4])."""
        maxit = self.p.maxit if maxit is None else maxit
        log = np.zeros((max(maxit, 1), 4))
        res = Result()
        _check(lib().sgpu_run(self._h, maxit, _dptr(log), print_every, C.byref(res)))
        return res, log[: res.iterations].copy()

    def download(self, field_id: int, out: np.ndarray | None = None) -> np.ndarray:
        """The field as an (nrows, ncols) array; into `out` (e.g. pinned host memory) if given."""
        if out is None:
            out = np.empty(self.shape)
        elif out.shape != self.shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of shape {self.shape}")
        _check(lib().sgpu_download(self._h, field_id, _dptr(out)))
        return out

    def upload(self, field_id: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"field shape {a.shape} != {self.shape}")
        _check(lib().sgpu_upload(self._h, field_id, _dptr(a)))

    def memory_bytes(self) -> int:
        n = C.c_size_t()
        _check(lib().sgpu_memory_bytes(self._h, C.byref(n)))
        return n.value

    def set_profiling(self, on) -> None:
        """False / True (every iteration timed per phase), or "sampled" (the first 10 iterations of a
        run timed, the rest replayed from the graph, phase times scaled to the run)."""
        mode = 2 if on == "sampled" else (1 if on else 0)
        _check(lib().sgpu_set_profiling(self._h, mode))

    def phase_seconds(self) -> dict:
        out = np.zeros(12)
        _check(lib().sgpu_phase_seconds(self._h, _dptr(out)))
        return dict(zip(PHASES, out.tolist()))

    def sweep_seconds(self) -> tuple[float, int]:
        """(device seconds, launches) of the streaming sweep kernels while profiling was on."""
        sec, n = C.c_double(), C.c_longlong()
        _check(lib().sgpu_sweep_seconds(self._h, C.byref(sec), C.byref(n)))
        return sec.value, n.value

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().sgpu_stream(self._h, C.byref(s)))
        return s.value or 0

    def attach_cnn(self, net: "Cnn | None", max_size: int = 256) -> None:
        """Use net as the p' warm start (not owned: keep it alive; None detaches)."""
        _check(lib().sgpu_attach_cnn(self._h, None if net is None else net._h, max_size))
        self._net = net  # keep the network alive while attached

    def load_cnn(self, path) -> None:
        _check(lib().sgpu_cnn_load(self._h, str(path).encode()))

    def set_mg_mode(self, tolerance: bool, pressure_tolerance: float = 1e-6, pressure_maxit: int = 1000) -> None:
        _check(lib().sgpu_set_mg_mode(self._h, 1 if tolerance else 0, pressure_tolerance, pressure_maxit))

    def warm_start_stats(self) -> dict:
        u, f, r = C.c_longlong(), C.c_longlong(), C.c_double()
        _check(lib().sgpu_warm_start_stats(self._h, C.byref(u), C.byref(f), C.byref(r)))
        return {"used": u.value, "fallbacks": f.value, "rel_initial": r.value}

    def cnn_sample(self, max_size: int = 256) -> tuple[np.ndarray, np.ndarray, int]:
        """Training pair from the last p' solve: (input (nx, ny, 2), target (nx, ny), level)."""
        nx, ny, lvl = C.c_int(), C.c_int(), C.c_int()
        _check(lib().sgpu_cnn_sample(self._h, max_size, None, None, C.byref(nx), C.byref(ny), C.byref(lvl)))
        x = np.empty((nx.value, ny.value, 2), np.float32)
        t = np.empty((nx.value, ny.value), np.float32)
        _check(lib().sgpu_cnn_sample(self._h, max_size, _fptr(x), _fptr(t), C.byref(nx), C.byref(ny),
                                     C.byref(lvl)))
        return x, t, lvl.value

    def last_solve_stats(self) -> dict:
        a, b, c, r = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        _check(lib().sgpu_last_solve_stats(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(r)))
        return {"cg_iterations": a.value, "mg_vcycles": b.value, "coarse_sweeps": c.value,
                "rel_residual": r.value}
