"""ctypes bindings of the checkers (test infrastructure only).

`Oracle` drives liborc.so, the C restatement of the reference's algorithm (oracle.c). `Reference`
drives _ref/libsimpleref.so, the reference's own C++ sources built where they lie; it exists only
where the reference tree was present at build time. `ReferenceGpu` drives _ref/libsimpleref_gpu.so,
the reference's own GPU backend (solver_hip.hip built as CUDA for sm_100a), the benchmark's reference
GPU baseline. Only tests/, __graft_entry__.smoke() and bench.py's reference legs import this module,
and only as the checker or a timed baseline.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORC_PATH = HERE / "liborc.so"
REF_PATH = HERE / "_ref" / "libsimpleref.so"
REFGPU_PATH = HERE / "_ref" / "libsimpleref_gpu.so"

_orc = None
_ref = None
_refgpu = None


def _params_type():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "sgpu", HERE.parent / "simple-hpc_b200" / "sgpu.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.Params


def orc_lib():
    global _orc
    if _orc is None:
        if not ORC_PATH.exists():
            raise ImportError(f"{ORC_PATH} is missing: run make -C oracle")
        L = C.CDLL(str(ORC_PATH))
        D, I, H = C.POINTER(C.c_double), C.c_int, C.c_void_p
        sig = {
            "orc_create": (H, [C.c_void_p]), "orc_destroy": (None, [H]),
            "orc_get": (I, [H, I, D]), "orc_set": (I, [H, I, D]),
            "orc_assemble_u": (None, [H]), "orc_bc_u": (None, [H]), "orc_residual_u": (C.c_double, [H]),
            "orc_sweep_u": (None, [H, I]), "orc_assemble_v": (None, [H]), "orc_bc_v": (None, [H]),
            "orc_residual_v": (C.c_double, [H]), "orc_sweep_v": (None, [H, I]),
            "orc_assemble_p": (C.c_double, [H]), "orc_solve_p": (None, [H]), "orc_correct": (None, [H]),
            "orc_outer_iteration": (None, [H, D]), "orc_run": (I, [H, I, D, C.POINTER(I)]),
            "orc_mg_level_dims": (I, [I, I, C.POINTER(I)]), "orc_mg_nlevels": (I, [H]),
            "orc_mg_last_coarse_sweeps": (I, [H]), "orc_cg_last_iterations": (I, [H]),
            "orc_cg_last_rel_residual": (C.c_double, [H]), "orc_mg_build": (None, [H]),
            "orc_mg_vcycle": (None, [H]), "orc_mg_get_level": (I, [H, I, I, D]),
            "orc_ordered_sum": (C.c_double, [D, I, I]),
            "orc_in_boundary_band": (I, [C.c_void_p, I, I]),
            "orc_convective": (None, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, I, I, D]),
            "orc_diffusive": (None, [C.c_void_p, I, I, D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _orc = L
    return _orc


def ref_available() -> bool:
    return REF_PATH.exists()


def ref_lib():
    global _ref
    if _ref is None:
        if not REF_PATH.exists():
            raise ImportError(f"{REF_PATH} is missing (the reference tree was not present at build time)")
        L = C.CDLL(str(REF_PATH))
        D, I, H = C.POINTER(C.c_double), C.c_int, C.c_void_p
        sig = {
            "ref_last_error": (C.c_char_p, []), "ref_make_params": (I, [C.c_char_p, C.POINTER(I), D]),
            "ref_create": (H, [C.c_char_p]), "ref_destroy": (None, [H]),
            "ref_set_threads": (None, [I]), "ref_max_threads": (I, []),
            "ref_get": (I, [H, I, D]), "ref_set": (I, [H, I, D]),
            "ref_assemble_u": (None, [H]), "ref_bc_u": (None, [H]), "ref_residual_u": (C.c_double, [H]),
            "ref_sweep_u": (None, [H, I]), "ref_assemble_v": (None, [H]), "ref_bc_v": (None, [H]),
            "ref_residual_v": (C.c_double, [H]), "ref_sweep_v": (None, [H, I]),
            "ref_assemble_p": (C.c_double, [H]), "ref_solve_p": (None, [H]), "ref_correct": (None, [H]),
            "ref_outer_iteration": (None, [H, D]),
            "ref_run": (I, [H, I, D, C.POINTER(I), D]),
            "ref_cg_last_iterations": (I, [H]), "ref_mg_last_coarse_sweeps": (I, [H]),
            "ref_write_outputs": (I, [H, C.c_char_p, I, D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _ref = L
    return _ref


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class _Base:
    """Shared phase interface of the two checkers."""

    prefix = ""

    def _f(self, name):
        return getattr(self._lib, f"{self.prefix}_{name}")

    def get(self, field_id: int) -> np.ndarray:
        out = np.empty(self.shape)
        if self._f("get")(self._h, field_id, _dp(out)) != 0:
            raise ValueError(f"bad field id {field_id}")
        return out

    def set(self, field_id: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.shape
        if self._f("set")(self._h, field_id, _dp(a)) != 0:
            raise ValueError(f"bad field id {field_id}")

    def assemble_u(self): self._f("assemble_u")(self._h)
    def bc_u(self): self._f("bc_u")(self._h)
    def residual_u(self) -> float: return self._f("residual_u")(self._h)
    def sweep_u(self, n: int): self._f("sweep_u")(self._h, n)
    def assemble_v(self): self._f("assemble_v")(self._h)
    def bc_v(self): self._f("bc_v")(self._h)
    def residual_v(self) -> float: return self._f("residual_v")(self._h)
    def sweep_v(self, n: int): self._f("sweep_v")(self._h, n)
    def assemble_p(self) -> float: return self._f("assemble_p")(self._h)
    def solve_p(self): self._f("solve_p")(self._h)
    def correct(self): self._f("correct")(self._h)

    def outer_iteration(self):
        r = np.zeros(3)
        self._f("outer_iteration")(self._h, _dp(r))
        return tuple(float(x) for x in r)

    def close(self):
        if getattr(self, "_h", None):
            self._f("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Oracle(_Base):
    """The C restatement (liborc.so) on one parameter set (an sgpu Params structure)."""

    prefix = "orc"

    def __init__(self, params):
        self._lib = orc_lib()
        self.params = params
        self.shape = (params.nrows, params.ncols)
        self._h = self._lib.orc_create(C.byref(params))

    def run(self, maxit: int):
        log = np.zeros((max(maxit, 1), 4))
        conv = C.c_int()
        n = self._lib.orc_run(self._h, maxit, _dp(log), C.byref(conv))
        return n, bool(conv.value), log[:n].copy()

    def cg_last_iterations(self) -> int:
        return self._lib.orc_cg_last_iterations(self._h)

    def mg_last_coarse_sweeps(self) -> int:
        return self._lib.orc_mg_last_coarse_sweeps(self._h)

    def mg_level(self, l: int, k: int, shape) -> np.ndarray:
        out = np.empty(shape)
        assert self._lib.orc_mg_get_level(self._h, l, k, _dp(out)) == 0
        return out


class Reference(_Base):
    """The reference's own C++ (oracle/_ref/libsimpleref.so), created from config text."""

    prefix = "ref"

    def __init__(self, config_text: str, shape):
        self._lib = ref_lib()
        self.shape = tuple(shape)
        self._h = self._lib.ref_create(config_text.encode())
        if not self._h:
            raise ValueError(self._lib.ref_last_error().decode())

    def run(self, maxit: int):
        log = np.zeros((max(maxit, 1), 4))
        conv = C.c_int()
        secs = C.c_double()
        n = self._lib.ref_run(self._h, maxit, _dp(log), C.byref(conv), C.byref(secs))
        return n, bool(conv.value), log[:n].copy()

    def cg_last_iterations(self) -> int:
        return self._lib.ref_cg_last_iterations(self._h)

    def mg_last_coarse_sweeps(self) -> int:
        return self._lib.ref_mg_last_coarse_sweeps(self._h)


def ordered_sum(values: np.ndarray) -> float:
    v = np.ascontiguousarray(values, dtype=np.float64)
    if v.ndim == 1:
        v = v.reshape(1, -1)
    return orc_lib().orc_ordered_sum(_dp(v), v.shape[0], v.shape[1])


def refgpu_available() -> bool:
    return REFGPU_PATH.exists()


def refgpu_lib():
    global _refgpu
    if _refgpu is None:
        if not REFGPU_PATH.exists():
            raise ImportError(f"{REFGPU_PATH} is missing (the reference tree or nvcc was not present at build time)")
        L = C.CDLL(str(REFGPU_PATH))
        D, I, H = C.POINTER(C.c_double), C.c_int, C.c_void_p
        for name, res, args in (("refgpu_last_error", C.c_char_p, []), ("refgpu_create", H, [C.c_char_p]),
                                ("refgpu_destroy", None, [H]), ("refgpu_iterations", I, [H, I, D, D]),
                                ("refgpu_run", I, [H, C.POINTER(I), C.POINTER(I), D]),
                                ("refgpu_download", I, [H, I, D])):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _refgpu = L
    return _refgpu


class ReferenceGpu:
    """The reference's own GPU backend (HipSolver built as CUDA) on one config, on device 0."""

    def __init__(self, config_text: str, shape):
        self._lib = refgpu_lib()
        self.shape = tuple(shape)
        self._h = self._lib.refgpu_create(config_text.encode())
        if not self._h:
            raise RuntimeError(self._lib.refgpu_last_error().decode())

    def iterations(self, n: int):
        """n outer iterations; returns (wall seconds, residuals[n, 3])."""
        res = np.zeros((max(n, 1), 3))
        secs = C.c_double()
        if self._lib.refgpu_iterations(self._h, n, _dp(res), C.byref(secs)) != 0:
            raise RuntimeError(self._lib.refgpu_last_error().decode())
        return secs.value, res[:n].copy()

    def run(self):
        """The reference's run_outer_loop to its tolerance or maxit: (iterations, converged, seconds)."""
        it, conv, secs = C.c_int(), C.c_int(), C.c_double()
        if self._lib.refgpu_run(self._h, C.byref(it), C.byref(conv), C.byref(secs)) != 0:
            raise RuntimeError(self._lib.refgpu_last_error().decode())
        return it.value, bool(conv.value), secs.value

    def get(self, field_id: int) -> np.ndarray:
        out = np.empty(self.shape)
        if self._lib.refgpu_download(self._h, field_id, _dp(out)) != 0:
            raise RuntimeError(self._lib.refgpu_last_error().decode())
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._lib.refgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
