"""ctypes binding of include/oco.h.

Mirrors the reference's interface for the hot path: calc_wavelength
(continuous_opacity.f90:37-62), pre_calc_opacity_quantities (:64-141, here
Engine.set_wavelengths) and the xy/lambda loop of flux_feautrier.f90:160-228
(Engine.solve_block for host arrays, Engine.solve_block_device for torch CUDA tensors).
Array shapes follow the reference's Fortran arrays read in C order:
  rho, T       (nx, ny, nz)          == Fortran (nz, ny, nx)
  U            (nw, nx, ny, nz+6)    == Fortran U(mz, ny, nx, nw)
  kappa, V     (nw, nx, ny, nz)
  Vtop, Vbot   (nw, nx, ny)          V at z index nz and 1
The device entry point also offers the lambda-fastest layout:
  U (nz+6, nx*ny, nw), kappa and V (nz, nx*ny, nw).
"""
import ctypes
import os
import weakref

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liboco_b200.so")

FORM_PLAIN, FORM_STABLE, FORM_MIXED = 0, 1, 2
LAYOUT_REFERENCE, LAYOUT_LAMBDA_FASTEST = 0, 1
_FORMS = {"plain": FORM_PLAIN, "stable": FORM_STABLE, "mixed": FORM_MIXED}

OCO_OK = 0
ERRORS = {-1: "EINVAL", -2: "ENOMEM", -3: "EZEROPIVOT", -4: "EGREY", -5: "ECUDA", -6: "ETIMEDOUT",
          -7: "EAGAIN", -8: "EADMIT", -9: "EIO", -10: "EDIM", -11: "ENOWAVES", -12: "ENAN", -13: "ECLOSED"}


class OcoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class OcoParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("nw", ctypes.c_int32),
                ("dz", ctypes.c_double), ("sigma_grey", ctypes.c_double), ("fully_ionized_T", ctypes.c_double),
                ("lgrey", ctypes.c_int32), ("form", ctypes.c_int32), ("layout", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class OcoBatchColumn(ctypes.Structure):
    """oco_batch_column: one column of a ragged batch (element offsets into the bound arrays)."""
    _fields_ = [("in_off", ctypes.c_int64), ("u_off", ctypes.c_int64), ("kv_off", ctypes.c_int64),
                ("flux_off", ctypes.c_int64), ("wave_off", ctypes.c_int64), ("nz", ctypes.c_int32),
                ("nw", ctypes.c_int32), ("dz", ctypes.c_double)]


class OcoBatchInfo(ctypes.Structure):
    _fields_ = [("ncol", ctypes.c_int64), ("npoints", ctypes.c_int64), ("max_nz", ctypes.c_int32),
                ("max_nw", ctypes.c_int32), ("tiling", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("tuned", ctypes.c_int32), ("ncandidates", ctypes.c_int32), ("cand_tiling", ctypes.c_int32 * 16),
                ("cand_blocks_per_sm", ctypes.c_int32 * 16), ("cand_ms", ctypes.c_double * 16),
                ("graph_launches", ctypes.c_int64)]


TILING_WARP_COLUMN, TILING_PACKED = 0, 1


class OcoServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("max_jobs", ctypes.c_int32), ("max_nz", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("budget_bytes", ctypes.c_double), ("chunk_points", ctypes.c_int64),
                ("reserve_bytes", ctypes.c_double)]


class OcoJob(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("nw", ctypes.c_int32),
                ("dz", ctypes.c_double), ("fully_ionized_T", ctypes.c_double), ("form", ctypes.c_int32),
                ("want_fields", ctypes.c_int32), ("rho", ctypes.c_void_p), ("T", ctypes.c_void_p),
                ("waves", ctypes.c_void_p)]


class OcoJobStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("error", ctypes.c_int32), ("inputs_consumed", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("bytes", ctypes.c_int64), ("submit_s", ctypes.c_double),
                ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double)]


JOB_STATES = ("queued", "running", "done", "failed")


class OcoDeckInfo(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("nw", ctypes.c_int32),
                ("nprocx", ctypes.c_int32), ("nprocy", ctypes.c_int32), ("nprocz", ctypes.c_int32),
                ("nxloc", ctypes.c_int32), ("nyloc", ctypes.c_int32), ("lgrey", ctypes.c_int32),
                ("lread_athena", ctypes.c_int32), ("reserved", ctypes.c_int32), ("dz", ctypes.c_double),
                ("sigma_grey", ctypes.c_double), ("fully_ionized_T", ctypes.c_double)]

class OcoDiskParams(ctypes.Structure):
    """oco_disk_params: the reference's synthetic disk (disk.f90:42-129) plus a seeded lognormal
    density perturbation."""
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("z0", ctypes.c_double), ("z1", ctypes.c_double), ("rho0", ctypes.c_double), ("H", ctypes.c_double),
                ("rho_floor", ctypes.c_double), ("midTemp", ctypes.c_double), ("sigma", ctypes.c_double),
                ("floorTemp", ctypes.c_double), ("isoTemp", ctypes.c_double), ("sigma_dex", ctypes.c_double),
                ("seed", ctypes.c_uint64)]


_LIB = None
_DP = ctypes.POINTER(ctypes.c_double)


def load_library(path=None):
    """Loads liboco_b200.so (built in-tree by ocotillo_b200.build).  Raises if absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m ocotillo_b200.build`")
    lib = ctypes.CDLL(path)
    V, I, P, D = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(OcoParams), ctypes.c_double
    sig = {
        "oco_abi_version": (I, []),
        "oco_create": (I, [ctypes.POINTER(V), I]),
        "oco_destroy": (None, [V]),
        "oco_last_error": (ctypes.c_char_p, [V]),
        "oco_calc_wavelength": (I, [D, D, ctypes.c_int32, _DP]),
        "oco_set_wavelengths": (I, [V, _DP, ctypes.c_int32]),
        "oco_solve_block": (I, [V, P, _DP, _DP, _DP, _DP, _DP, _DP, _DP]),
        "oco_solve_block_device": (I, [V, P, V, V, V, V, V, V, V, V]),
        "oco_synchronize": (I, [V]),
        "oco_set_mixed_repair": (I, [V, D]),
        "oco_disk_inputs": (I, [ctypes.POINTER(OcoDiskParams), _DP, _DP, _DP]),
        "oco_deck_block_inputs_device": (I, [V, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.POINTER(OcoDeckInfo), V, V, _DP, _DP, V]),
        "oco_disk_inputs_device": (I, [V, ctypes.POINTER(OcoDiskParams), V, V, V]),
        "oco_mixed_repairs": (I, [V, ctypes.POINTER(ctypes.c_int64)]),
        "oco_kernel_launches": (ctypes.c_int64, [V]),
        "oco_check_bounded_wait": (I, [V, ctypes.c_int64]),
        "oco_integrated_flux_device": (I, [V, P, V, V, V]),
        "oco_intensities_device": (I, [V, P, V, V, V, V, V]),
        "oco_optical_depth_device": (I, [V, P, V, V, D, V, V, V]),
        "oco_set_profiling": (I, [V, I]),
        "oco_kernel_times": (I, [V, _DP, _DP, ctypes.POINTER(ctypes.c_int64)]),
        "oco_solve_block_noalloc": (I, [P, _DP, V, V, V, V, V, V, V, V]),
        "oco_noalloc_last_error": (ctypes.c_char_p, []),
        "oco_batch_create": (I, [V, ctypes.POINTER(OcoBatchColumn), ctypes.c_int64, _DP, ctypes.c_int64,
                                 ctypes.c_int32, ctypes.c_int32, D, ctypes.POINTER(V)]),
        "oco_batch_bind": (I, [V, V, V, ctypes.c_int64, V, ctypes.c_int64, V, V, ctypes.c_int64, V, V,
                               ctypes.c_int64]),
        "oco_batch_tune": (I, [V]),
        "oco_batch_set_tiling": (I, [V, ctypes.c_int32, ctypes.c_int32]),
        "oco_batch_run": (I, [V, V]),
        "oco_batch_wait": (I, [V]),
        "oco_batch_get_info": (I, [V, ctypes.POINTER(OcoBatchInfo)]),
        "oco_batch_destroy": (None, [V]),
        "oco_server_create": (I, [ctypes.POINTER(OcoServerConfig), ctypes.POINTER(V)]),
        "oco_server_submit": (I, [V, ctypes.POINTER(OcoJob), ctypes.POINTER(ctypes.c_int64)]),
        "oco_server_status": (I, [V, ctypes.c_int64, ctypes.POINTER(OcoJobStatus)]),
        "oco_server_wait": (I, [V, ctypes.c_int64, D]),
        "oco_server_fetch": (I, [V, ctypes.c_int64, _DP, _DP, _DP, _DP, _DP]),
        "oco_server_destroy": (None, [V]),
        "oco_server_last_error": (ctypes.c_char_p, []),
        "oco_deck_block_inputs": (I, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.POINTER(OcoDeckInfo), _DP, _DP, _DP, _DP]),
        "oco_run_deck": (I, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                             ctypes.c_int32]),
        "oco_format_e": (None, [D, ctypes.c_int32, ctypes.c_int32, ctypes.c_char_p]),
        "oco_deck_last_error": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIB = lib
    return lib


def _ptr(a):
    if a is None:
        return None
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("need a C-contiguous float64 numpy array")
    return a.ctypes.data_as(_DP)


def _need_host(name, a, numel):
    """A host array handed to the library: C-contiguous float64 of exactly numel elements (a
    shorter one would be read or written past its end)."""
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError(f"{name}: need a C-contiguous float64 numpy array")
    if a.size != numel:
        raise ValueError(f"{name}: {a.size} elements where the block has {numel}")


def _need_tensor(name, t, numel, device, dtype=None):
    """A device array handed to a kernel: a contiguous CUDA tensor of exactly numel elements of
    dtype (float64 by default) on the context's device.  A wrong size would let the kernel read
    or write past the caller's allocation, so it is refused here, before anything is launched."""
    import torch
    dtype = dtype or torch.float64
    if t.numel() != numel:
        raise ValueError(f"{name}: {t.numel()} elements where the block has {numel}")
    if t.dtype != dtype or not t.is_contiguous():
        raise ValueError(f"{name}: need a contiguous {dtype} tensor")
    if not t.is_cuda or t.device.index != int(device):
        raise ValueError(f"{name}: need a tensor on cuda:{int(device)}")


def format_e(v, w=15, d=5):
    """gfortran Ew.d editing (io.f90's e15.5 fields)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(w + 1)
    lib.oco_format_e(float(v), int(w), int(d), buf)
    return buf.value.decode()


def deck_block_inputs(deck_dir, snapshot="0000", iprocx=0, iprocy=0):
    """Inputs of processor block (iprocx, iprocy) of a reference deck (synthetic disk or Athena
    reader), host only: dict with info fields, rho and T (nxloc, nyloc, nz), wa, z (nz+6)."""
    lib = load_library()
    info = OcoDeckInfo()
    rc = lib.oco_deck_block_inputs(deck_dir.encode(), snapshot.encode(), 0, 0, ctypes.byref(info), None, None,
                                   None, None)
    if rc:
        raise OcoError(rc, lib.oco_deck_last_error().decode())
    rho = np.empty((info.nxloc, info.nyloc, info.nz))
    T = np.empty_like(rho)
    wa = np.empty(info.nw)
    z = np.empty(info.nz + 6)
    rc = lib.oco_deck_block_inputs(deck_dir.encode(), snapshot.encode(), int(iprocx), int(iprocy),
                                   ctypes.byref(info), _ptr(rho), _ptr(T), _ptr(wa), _ptr(z))
    if rc:
        raise OcoError(rc, lib.oco_deck_last_error().decode())
    out = {k: getattr(info, k) for k, _ in OcoDeckInfo._fields_}
    out.update(rho=rho, T=T, wa=wa, z=z)
    return out


def run_deck(deck_dir, snapshot="0000", out_dir=None, form="plain", device=0, write_binary=True):
    """Runs a reference deck with the loop on the GPU; writes diagnostics.txt, the grids and
    (write_binary) the per-block Fortran unformatted files into out_dir (default
    deck_dir/output).  Returns the return code (0, or -3 where the reference stops on a zero
    pivot); raises on other errors."""
    lib = load_library()
    rc = lib.oco_run_deck(deck_dir.encode(), snapshot.encode(), (out_dir or "").encode(),
                          _FORMS[form] if isinstance(form, str) else int(form), int(device), int(bool(write_binary)))
    if rc and rc != -3:
        raise OcoError(rc, lib.oco_deck_last_error().decode())
    return rc


def read_fortran_records(path):
    """Records of a Fortran unformatted sequential file (gfortran markers and subrecords) as
    a list of bytes objects."""
    data = open(path, "rb").read()
    recs, pos, cur = [], 0, b""
    while pos < len(data):
        lead = int.from_bytes(data[pos:pos + 4], "little", signed=True)
        n = abs(lead)
        cur += data[pos + 4:pos + 4 + n]
        pos += 8 + n
        if lead >= 0:
            recs.append(cur)
            cur = b""
    return recs


def calc_wavelength(w1, w0, nw):
    """Linear grid of continuous_opacity.f90:37-62 (argument order as there)."""
    lib = load_library()
    wa = np.empty(max(int(nw), 0))  # nw < 1 reaches the library's check (OCO_EINVAL)
    rc = lib.oco_calc_wavelength(float(w1), float(w0), int(nw), _ptr(wa))
    if rc:
        raise OcoError(rc, lib.oco_last_error(None).decode())
    return wa


class Engine:
    """One context of the engine on one CUDA device."""

    def __init__(self, device=0):
        self.lib = load_library()
        self.ctx = ctypes.c_void_p()
        rc = self.lib.oco_create(ctypes.byref(self.ctx), int(device))
        if rc:
            raise OcoError(rc, self.lib.oco_last_error(None).decode())
        self.device = device
        self.nw = 0
        self._batches = weakref.WeakSet()  # a batch refers to this context: closed before it

    def close(self):
        for b in list(getattr(self, "_batches", ())):
            b.close()
        if self.ctx:
            self.lib.oco_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise OcoError(rc, self.lib.oco_last_error(self.ctx).decode())

    def set_wavelengths(self, wa):
        """pre_calc_opacity_quantities for a wavelength grid in Angstrom."""
        wa = np.ascontiguousarray(np.atleast_1d(wa), dtype=np.float64)
        self._check(self.lib.oco_set_wavelengths(self.ctx, _ptr(wa), wa.size))
        self.nw = wa.size

    def params(self, shape, nw, dz, fully_ionized_T=2e4, lgrey=False, sigma_grey=0.4, form="plain",
               layout=LAYOUT_REFERENCE):
        nx, ny, nz = shape
        return OcoParams(nx, ny, nz, nw, float(dz), float(sigma_grey), float(fully_ionized_T), int(bool(lgrey)),
                         _FORMS[form] if isinstance(form, str) else int(form), int(layout), 0)

    def solve_block(self, rho, T, dz, fully_ionized_T=2e4, lgrey=False, sigma_grey=0.4, form="plain",
                    want=("U", "kappa", "V", "Vtop", "Vbot"), out=None, allow_zero_pivot=False):
        """The reference's xy/lambda loop on host arrays.  rho, T: (nx, ny, nz) float64.
        Returns a dict of numpy arrays (reference layout).  `out` may supply preallocated
        (e.g. pinned) arrays by name.  An exactly zero Thomas pivot raises OcoError
        (EZEROPIVOT), as the reference stops there; with allow_zero_pivot=True the results
        are returned with out['zero_pivot'] = True instead."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        if rho.ndim != 3 or T.shape != rho.shape:
            raise ValueError(f"rho and T: need one shape (nx, ny, nz), got {rho.shape} and {T.shape}")
        nx, ny, nz = rho.shape
        nw = 1 if lgrey else self.nw
        out = dict(out or {})
        shapes = {"U": (nw, nx, ny, nz + 6), "kappa": (nw, nx, ny, nz), "V": (nw, nx, ny, nz),
                  "Vtop": (nw, nx, ny), "Vbot": (nw, nx, ny)}
        for k in set(want):
            if k not in out:
                out[k] = np.empty(shapes[k])
        if nw >= 1:  # without wavelength tables the library reports OCO_ENOWAVES
            for k in shapes:
                if out.get(k) is not None:
                    _need_host(k, out[k], int(np.prod(shapes[k])))
        prm = self.params(rho.shape, nw, dz, fully_ionized_T, lgrey, sigma_grey, form)
        rc = self.lib.oco_solve_block(self.ctx, ctypes.byref(prm), _ptr(rho), _ptr(T), _ptr(out.get("U")),
                                      _ptr(out.get("kappa")), _ptr(out.get("V")), _ptr(out.get("Vtop")),
                                      _ptr(out.get("Vbot")))
        out["zero_pivot"] = rc == -3
        if not (rc == -3 and allow_zero_pivot):
            self._check(rc)
        return out

    def solve_block_device(self, rho, T, dz, out, fully_ionized_T=2e4, lgrey=False, sigma_grey=0.4,
                           form="plain", layout=LAYOUT_REFERENCE, stream=None):
        """Same loop on torch CUDA tensors (float64, contiguous), enqueued on `stream`
        (default: torch's current stream).  `out` maps any of 'U', 'kappa', 'V', 'Vtop', 'Vbot'
        to preallocated tensors of the layout's shapes (absent names are not stored)."""
        import torch
        if rho.dim() != 3:
            raise ValueError(f"rho: need shape (nx, ny, nz), got {tuple(rho.shape)}")
        nx, ny, nz = rho.shape
        nw = 1 if lgrey else self.nw
        cols = nx * ny
        _need_tensor("rho", rho, cols * nz, self.device)
        _need_tensor("T", T, cols * nz, self.device)
        sizes = {"U": nw * cols * (nz + 6), "kappa": nw * cols * nz, "V": nw * cols * nz, "Vtop": nw * cols,
                 "Vbot": nw * cols}
        for k, v in out.items():
            if k not in sizes:
                raise ValueError(f"out: unknown array {k!r} (U, kappa, V, Vtop, Vbot)")
            if v is not None and nw >= 1:  # without wavelength tables the library reports OCO_ENOWAVES
                _need_tensor(k, v, sizes[k], self.device)
        if stream is None:
            stream = torch.cuda.current_stream(rho.device)
        prm = self.params(rho.shape, nw, dz, fully_ionized_T, lgrey, sigma_grey, form, layout)

        def p(name):
            t = out.get(name)
            return ctypes.c_void_p(t.data_ptr()) if t is not None else None

        rc = self.lib.oco_solve_block_device(self.ctx, ctypes.byref(prm), ctypes.c_void_p(rho.data_ptr()),
                                             ctypes.c_void_p(T.data_ptr()), p("U"), p("kappa"), p("V"),
                                             p("Vtop"), p("Vbot"), ctypes.c_void_p(stream.cuda_stream))
        self._check(rc)
        return out

    def synchronize(self):
        self._check(self.lib.oco_synchronize(self.ctx))

    def set_mixed_repair(self, cond_max=100.0):
        """Condition number of a mixed-form emergent flux above which the item is re-solved in the
        stable FP64 form (float('inf') turns the re-solve off)."""
        self._check(self.lib.oco_set_mixed_repair(self.ctx, min(float(cond_max), 3.4e38)))

    def disk_inputs_device(self, rho, T, disk, stream=None):
        """Fills torch CUDA float64 tensors rho, T of shape (nx, ny, nz) with the synthetic disk of
        `disk` (a dict of disk_params' keys), on the device; returns dz."""
        import torch
        prm = disk_params(tuple(rho.shape), **disk)
        n = rho.numel()
        _need_tensor("rho", rho, n, self.device)
        _need_tensor("T", T, n, self.device)
        if stream is None:
            stream = torch.cuda.current_stream(rho.device)
        self._check(self.lib.oco_disk_inputs_device(self.ctx, ctypes.byref(prm), ctypes.c_void_p(rho.data_ptr()),
                                                     ctypes.c_void_p(T.data_ptr()),
                                                     ctypes.c_void_p(stream.cuda_stream)))
        return (prm.z1 - prm.z0) / (prm.nz - 1)

    def deck_block_inputs_device(self, deck_dir, snapshot="0000", iprocx=0, iprocy=0, stream=None):
        """Inputs of processor block (iprocx, iprocy) of a reference deck delivered into device
        memory (an Athena snapshot goes from disk to HBM): dict with info fields, rho and T as
        torch CUDA tensors (nxloc, nyloc, nz), wa and z (numpy)."""
        import torch
        info = OcoDeckInfo()
        rc = self.lib.oco_deck_block_inputs(deck_dir.encode(), snapshot.encode(), 0, 0, ctypes.byref(info), None, None,
                                            None, None)
        if rc:
            raise OcoError(rc, self.lib.oco_deck_last_error().decode())
        dev = torch.device("cuda", self.device)
        rho = torch.empty((info.nxloc, info.nyloc, info.nz), dtype=torch.float64, device=dev)
        T = torch.empty_like(rho)
        wa = np.empty(info.nw)
        z = np.empty(info.nz + 6)
        if stream is None:
            stream = torch.cuda.current_stream(dev)
        rc = self.lib.oco_deck_block_inputs_device(self.ctx, deck_dir.encode(), snapshot.encode(), int(iprocx),
                                                   int(iprocy), ctypes.byref(info), ctypes.c_void_p(rho.data_ptr()),
                                                   ctypes.c_void_p(T.data_ptr()), _ptr(wa), _ptr(z),
                                                   ctypes.c_void_p(stream.cuda_stream))
        if rc:
            raise OcoError(rc, self.lib.oco_deck_last_error().decode())
        out = {k: getattr(info, k) for k, _ in OcoDeckInfo._fields_}
        out.update(rho=rho, T=T, wa=wa, z=z)
        return out

    def mixed_repairs(self):
        """Items the mixed form re-solved in FP64 since the previous call (waits for the work)."""
        n = ctypes.c_int64(0)
        self._check(self.lib.oco_mixed_repairs(self.ctx, ctypes.byref(n)))
        return n.value

    def intensities_device(self, U, V, shape, nw, out, layout=LAYOUT_REFERENCE, stream=None):
        """Ip = U + V, Im = U - V (calc_intensity) on torch CUDA tensors of a solved block of
        shape (nx, ny, nz) with nw wavelengths; `out` maps 'Ip' and/or 'Im' to tensors shaped
        like V."""
        import torch
        nx, ny, nz = shape
        n = nw * nx * ny * nz
        _need_tensor("U", U, nw * nx * ny * (nz + 6), self.device)
        _need_tensor("V", V, n, self.device)
        for k in ("Ip", "Im"):
            if out.get(k) is not None:
                _need_tensor(k, out[k], n, self.device)
        if stream is None:
            stream = torch.cuda.current_stream(U.device)
        prm = self.params(shape, nw, 1.0, layout=layout)
        p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
        self._check(self.lib.oco_intensities_device(self.ctx, ctypes.byref(prm), p(U), p(V), p(out.get("Ip")),
                                                    p(out.get("Im")), ctypes.c_void_p(stream.cuda_stream)))
        return out

    def optical_depth_device(self, kappa, rho, dz, target_tau=1.0, tau=None, photo=None, layout=LAYOUT_REFERENCE,
                             stream=None):
        """tau = cumsum_z(kappa rho dz) and the photosphere index (first z with tau >= target,
        -1 if none) on torch CUDA tensors of a solved block; rho (nx, ny, nz)."""
        import torch
        if rho.dim() != 3:
            raise ValueError(f"rho: need shape (nx, ny, nz), got {tuple(rho.shape)}")
        nx, ny, nz = rho.shape
        nw = kappa.numel() // (nx * ny * nz)
        if nw < 1 or kappa.numel() != nw * nx * ny * nz:
            raise ValueError(f"kappa: {kappa.numel()} elements is not nw * {nx * ny * nz} for the block of rho")
        _need_tensor("kappa", kappa, kappa.numel(), self.device)
        _need_tensor("rho", rho, nx * ny * nz, self.device)
        if tau is not None:
            _need_tensor("tau", tau, kappa.numel(), self.device)
        if photo is not None:
            _need_tensor("photo", photo, nw * nx * ny, self.device, dtype=torch.int32)
        if stream is None:
            stream = torch.cuda.current_stream(kappa.device)
        prm = self.params((nx, ny, nz), nw, dz, layout=layout)
        p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
        self._check(self.lib.oco_optical_depth_device(self.ctx, ctypes.byref(prm), p(kappa), p(rho), float(target_tau),
                                                      p(tau), p(photo), ctypes.c_void_p(stream.cuda_stream)))

    def integrated_flux_device(self, V, shape, out=None, stream=None):
        """Wavelength-integrated emergent flux (trapezoid rule over the context's wavelength
        grid, lambda in cm) of an emergent-flux plane V (nw, nx, ny) on the device, as a
        (nx, ny) float64 tensor."""
        import torch
        nx, ny = shape[0], shape[1]
        nw = V.numel() // (nx * ny)
        if nw < 1 or V.numel() != nw * nx * ny:
            raise ValueError(f"V: {V.numel()} elements is not nw * {nx * ny} for a ({nx}, {ny}) plane")
        _need_tensor("V", V, V.numel(), self.device)
        if out is None:
            out = torch.empty((nx, ny), dtype=torch.float64, device=V.device)
        _need_tensor("out", out, nx * ny, self.device)
        if stream is None:
            stream = torch.cuda.current_stream(V.device)
        prm = self.params((nx, ny, 2), nw, 1.0)
        self._check(self.lib.oco_integrated_flux_device(self.ctx, ctypes.byref(prm), ctypes.c_void_p(V.data_ptr()),
                                                        ctypes.c_void_p(out.data_ptr()),
                                                        ctypes.c_void_p(stream.cuda_stream)))
        return out

    def check_bounded_wait(self, spin_limit=100):
        """Return code of the bounded-wait diagnostic (OCO_ETIMEDOUT = -6 expected)."""
        return self.lib.oco_check_bounded_wait(self.ctx, int(spin_limit))

    @property
    def kernel_launches(self):
        return self.lib.oco_kernel_launches(self.ctx)

    def set_profiling(self, enable=True):
        self._check(self.lib.oco_set_profiling(self.ctx, int(bool(enable))))

    def kernel_times(self):
        """(solve_ms, pillars_ms, solve_launches) since the last call (profiling on)."""
        a, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        self._check(self.lib.oco_kernel_times(self.ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(n)))
        return a.value, b.value, n.value

    def batch(self, nz, nw, dz, waves, wave_off, layout=LAYOUT_LAMBDA_FASTEST, fully_ionized_T=2e4, form="mixed",
              offsets=None):
        """A ragged batch of len(nz) columns: column i has nz[i] levels, spacing dz[i] and the
        nw[i] wavelengths waves[wave_off[i]:...]; form is "plain", "stable" or "mixed".  The
        arrays are packed densely (dense_batch_offsets) unless offsets gives the per-column
        element offsets {"in_off", "u_off", "kv_off", "flux_off"} of the caller's packing."""
        return Batch(self, nz, nw, dz, waves, wave_off, layout, fully_ionized_T, form, offsets)


DISK_DEFAULTS = {"z0": -5e15, "z1": 5e15, "rho0": 1e-9, "H": 1.496e14, "rho_floor": 1e-24, "midTemp": 6.1e4,
                 "sigma": 2.5e14, "floorTemp": 2000.0, "isoTemp": 1e8, "sigma_dex": 0.0, "seed": 0}


def disk_params(shape, **kw):
    """oco_disk_params for a block of shape (nx, ny, nz); keys as in DISK_DEFAULTS (the AGN grid's
    disk: the Gaussian temperature applies since isoTemp exceeds midTemp)."""
    nx, ny, nz = shape
    d = dict(DISK_DEFAULTS, **kw)
    unknown = set(kw) - set(DISK_DEFAULTS)
    if unknown:
        raise ValueError(f"disk parameters: unknown {sorted(unknown)}")
    return OcoDiskParams(int(nx), int(ny), int(nz), 0, *(float(d[k]) for k in
                                                          ("z0", "z1", "rho0", "H", "rho_floor", "midTemp", "sigma",
                                                           "floorTemp", "isoTemp", "sigma_dex")), int(d["seed"]))


def disk_inputs(shape, **kw):
    """Host arrays rho, T (nx, ny, nz) and dz of the synthetic disk (bit-identical to
    Engine.disk_inputs_device); no GPU needed."""
    lib = load_library()
    prm = disk_params(shape, **kw)
    rho, T = np.empty(shape), np.empty(shape)
    dz = ctypes.c_double()
    rc = lib.oco_disk_inputs(ctypes.byref(prm), _ptr(rho), _ptr(T), ctypes.byref(dz))
    if rc:
        raise OcoError(rc, lib.oco_last_error(None).decode())
    return rho, T, dz.value


def dense_batch_offsets(nz, nw):
    """Dense packing of a batch's arrays: per column in_off (rho, T), u_off (U),
    kv_off (kappa, V), flux_off (Vtop, Vbot), and the total element counts of each."""
    nz = np.asarray(nz, dtype=np.int64)
    nw = np.asarray(nw, dtype=np.int64)

    def pre(x):
        return np.concatenate([[0], np.cumsum(x)])

    p_in, p_u, p_kv, p_f = pre(nz), pre((nz + 6) * nw), pre(nz * nw), pre(nw)
    return {"in_off": p_in[:-1], "u_off": p_u[:-1], "kv_off": p_kv[:-1], "flux_off": p_f[:-1],
            "n_in": int(p_in[-1]), "n_u": int(p_u[-1]), "n_kv": int(p_kv[-1]), "n_flux": int(p_f[-1])}


def batch_offsets(nz, nw, in_off, u_off, kv_off, flux_off):
    """A caller's packing of a batch's arrays in the form dense_batch_offsets returns: the
    per-column offsets and, per array, the element count that holds every column's range."""
    nz = np.asarray(nz, dtype=np.int64)
    nw = np.asarray(nw, dtype=np.int64)
    o = {k: np.asarray(v, dtype=np.int64).copy() for k, v in
         (("in_off", in_off), ("u_off", u_off), ("kv_off", kv_off), ("flux_off", flux_off))}
    if any(v.shape != nz.shape for v in o.values()):
        raise ValueError("batch_offsets: one offset per column")
    o["n_in"] = int((o["in_off"] + nz).max())
    o["n_u"] = int((o["u_off"] + (nz + 6) * nw).max())
    o["n_kv"] = int((o["kv_off"] + nz * nw).max())
    o["n_flux"] = int((o["flux_off"] + nw).max())
    return o


class Batch:
    """Ragged batch (include/oco.h, oco_batch_*): independent columns of different nz, dz
    and wavelength grids, solved by one persistent launch replayed as a CUDA graph.  Arrays
    are torch CUDA float64 tensors packed as dense_batch_offsets describes (or as the caller's
    offsets give, see batch_offsets); per column U is [z][lambda] (LAYOUT_LAMBDA_FASTEST) or
    [lambda][z] (LAYOUT_REFERENCE)."""

    def __init__(self, eng, nz, nw, dz, waves, wave_off, layout, fully_ionized_T, form, offsets=None):
        self.eng, self.lib = eng, eng.lib
        n = len(nz)
        self.nz = np.asarray(nz, dtype=np.int64)
        self.nw = np.asarray(nw, dtype=np.int64)
        if offsets is None:
            self.offsets = dense_batch_offsets(self.nz, self.nw)
        else:
            self.offsets = batch_offsets(self.nz, self.nw, offsets["in_off"], offsets["u_off"], offsets["kv_off"],
                                         offsets["flux_off"])
        cols = (OcoBatchColumn * n)()
        o = self.offsets
        for i in range(n):
            cols[i] = OcoBatchColumn(int(o["in_off"][i]), int(o["u_off"][i]), int(o["kv_off"][i]),
                                     int(o["flux_off"][i]), int(wave_off[i]), int(self.nz[i]), int(self.nw[i]),
                                     float(dz[i]))
        w = np.ascontiguousarray(waves, dtype=np.float64)
        self.layout = layout
        self.h = ctypes.c_void_p()
        rc = self.lib.oco_batch_create(eng.ctx, cols, n, _ptr(w), w.size,
                                       _FORMS[form] if isinstance(form, str) else int(form), int(layout),
                                       float(fully_ionized_T), ctypes.byref(self.h))
        eng._check(rc)
        self.arrays = None
        eng._batches.add(self)

    def alloc(self, device="cuda", want=("U", "kappa", "V", "Vtop", "Vbot")):
        """Allocates output tensors of the dense packing."""
        import torch
        o = self.offsets
        n = {"U": o["n_u"], "kappa": o["n_kv"], "V": o["n_kv"], "Vtop": o["n_flux"], "Vbot": o["n_flux"]}
        return {k: torch.empty(n[k], dtype=torch.float64, device=device) for k in want}

    def bind(self, rho, T, out):
        """Binds device inputs (dense rho, T) and outputs (dict of U, kappa, V, Vtop, Vbot).
        The library checks every column's range against the element counts passed here; the
        arrays themselves must be float64 CUDA tensors on the engine's device."""
        for k in out:
            if k not in ("U", "kappa", "V", "Vtop", "Vbot"):
                raise ValueError(f"out: unknown array {k!r} (U, kappa, V, Vtop, Vbot)")
        for name, t in (("rho", rho), ("T", T)) + tuple(out.items()):
            if t is not None:
                _need_tensor(name, t, t.numel(), self.eng.device)
        o = self.offsets

        def p(t):
            return ctypes.c_void_p(t.data_ptr()) if t is not None else None

        g = out.get
        n_kv = (g("kappa") if g("kappa") is not None else g("V"))
        n_fl = (g("Vtop") if g("Vtop") is not None else g("Vbot"))
        rc = self.lib.oco_batch_bind(self.h, p(rho), p(T), min(rho.numel(), T.numel()), p(g("U")),
                                     g("U").numel() if g("U") is not None else 0, p(g("kappa")), p(g("V")),
                                     n_kv.numel() if n_kv is not None else 0, p(g("Vtop")), p(g("Vbot")),
                                     n_fl.numel() if n_fl is not None else 0)
        self.eng._check(rc)
        self.arrays = (rho, T, out)
        return out

    def tune(self):
        self.eng._check(self.lib.oco_batch_tune(self.h))
        return self.info()

    def set_tiling(self, tiling, blocks_per_sm=0):
        """tiling: 'warp_column' or 'packed' (or TILING_*); blocks_per_sm 0 = occupancy limit."""
        t = {"warp_column": TILING_WARP_COLUMN, "packed": TILING_PACKED}.get(tiling, tiling)
        self.eng._check(self.lib.oco_batch_set_tiling(self.h, int(t), int(blocks_per_sm)))

    def run(self, stream=None):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream()
        self.eng._check(self.lib.oco_batch_run(self.h, ctypes.c_void_p(stream.cuda_stream)))

    def wait(self):
        self.eng._check(self.lib.oco_batch_wait(self.h))

    def info(self):
        inf = OcoBatchInfo()
        self.eng._check(self.lib.oco_batch_get_info(self.h, ctypes.byref(inf)))
        n = inf.ncandidates
        return {"ncol": inf.ncol, "npoints": inf.npoints, "max_nz": inf.max_nz, "max_nw": inf.max_nw,
                "tiling": ("warp_column", "packed")[inf.tiling], "blocks_per_sm": inf.blocks_per_sm,
                "tuned": bool(inf.tuned), "graph_launches": inf.graph_launches,
                "candidates": [{"tiling": ("warp_column", "packed")[inf.cand_tiling[i]],
                                "blocks_per_sm": inf.cand_blocks_per_sm[i], "ms": inf.cand_ms[i]}
                               for i in range(n)]}

    def column(self, out, i, name):
        """View of column i's block of output `name` as (nz+6, nw) / (nz, nw) / (nw,) in z, lambda
        order (whatever the layout)."""
        o = self.offsets
        nz, nw = int(self.nz[i]), int(self.nw[i])
        if name == "U":
            a = out["U"][o["u_off"][i]:o["u_off"][i] + (nz + 6) * nw]
            rows = nz + 6
        elif name in ("kappa", "V"):
            a = out[name][o["kv_off"][i]:o["kv_off"][i] + nz * nw]
            rows = nz
        else:
            return out[name][o["flux_off"][i]:o["flux_off"][i] + nw]
        return a.view(rows, nw) if self.layout == LAYOUT_LAMBDA_FASTEST else a.view(nw, rows).t()

    def close(self):
        if self.h:
            self.lib.oco_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop (include/oco.h, oco_server_*): jobs (a block of columns plus its wavelength
    grid) are admitted as job slots and device memory free up, and their launches overlap on
    the device.  Inputs are numpy float64 arrays (nx, ny, nz) or torch CUDA float64 tensors of
    that shape; results come back as numpy arrays in the reference layout."""

    def __init__(self, device=0, max_jobs=4, max_nz=0, budget_bytes=0.0, chunk_points=0, reserve_bytes=0.0):
        self.lib = load_library()
        self.h = ctypes.c_void_p()
        cfg = OcoServerConfig(int(device), int(max_jobs), int(max_nz), 0, float(budget_bytes), int(chunk_points),
                              float(reserve_bytes))
        self._check(self.lib.oco_server_create(ctypes.byref(cfg), ctypes.byref(self.h)))
        self._jobs = {}

    def _check(self, rc):
        if rc:
            raise OcoError(rc, self.lib.oco_server_last_error().decode())

    @staticmethod
    def _addr(name, a):
        if isinstance(a, np.ndarray):
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError(f"{name}: need a C-contiguous float64 numpy array")
            return a.ctypes.data
        if not (getattr(a, "is_cuda", False) and a.is_contiguous() and str(a.dtype) == "torch.float64"):
            raise ValueError(f"{name}: need a C-contiguous float64 numpy array or contiguous float64 CUDA tensor")
        return a.data_ptr()

    def submit(self, rho, T, waves, dz, form="mixed", fully_ionized_T=2e4, want_fields=False):
        """Queues a job; returns its id.  rho and T are referenced until the job is fetched."""
        if len(rho.shape) != 3 or tuple(T.shape) != tuple(rho.shape):
            raise ValueError(f"rho and T: need one shape (nx, ny, nz), got {tuple(rho.shape)} and {tuple(T.shape)}")
        nx, ny, nz = rho.shape
        w = np.ascontiguousarray(np.atleast_1d(waves), dtype=np.float64)
        job = OcoJob(nx, ny, nz, w.size, float(dz), float(fully_ionized_T),
                     _FORMS[form] if isinstance(form, str) else int(form), int(bool(want_fields)),
                     self._addr("rho", rho), self._addr("T", T), w.ctypes.data)
        jid = ctypes.c_int64()
        self._check(self.lib.oco_server_submit(self.h, ctypes.byref(job), ctypes.byref(jid)))
        self._jobs[jid.value] = (rho, T, (nx, ny, nz, w.size), bool(want_fields))
        return jid.value

    def submit_deck(self, eng, deck_dir, snapshot="0000", iprocx=0, iprocy=0, form="mixed", want_fields=False):
        """Queues processor block (iprocx, iprocy) of a reference deck as a job: its snapshot is
        read into HBM (Engine.deck_block_inputs_device on `eng`, the server's device) and the job
        takes the device arrays.  Returns (job id, the block's info dict)."""
        d = eng.deck_block_inputs_device(deck_dir, snapshot, iprocx, iprocy)
        jid = self.submit(d["rho"], d["T"], d["wa"], d["dz"], form=form, fully_ionized_T=d["fully_ionized_T"],
                          want_fields=want_fields)
        return jid, d

    def status(self, jid):
        st = OcoJobStatus()
        self._check(self.lib.oco_server_status(self.h, int(jid), ctypes.byref(st)))
        return {"state": JOB_STATES[st.state], "error": st.error, "inputs_consumed": bool(st.inputs_consumed),
                "bytes": st.bytes, "submit_s": st.submit_s, "admit_s": st.admit_s, "done_s": st.done_s}

    def wait(self, jid, timeout=3600.0):
        self._check(self.lib.oco_server_wait(self.h, int(jid), float(timeout)))

    def fetch(self, jid, fields=None, out=None):
        """Results of a done job as numpy arrays: Vtop, Vbot (nw, nx, ny) and, if the job kept
        them (or fields=True), U (nw, nx, ny, nz+6), kappa and V (nw, nx, ny, nz).  `out` may
        supply the destination arrays by name (e.g. views of pinned memory; C-contiguous
        float64 with exactly those element counts).  Releases the job."""
        _, _, (nx, ny, nz, nw), kept = self._jobs[jid]
        fields = kept if fields is None else fields
        shapes = {"Vtop": (nw, nx, ny), "Vbot": (nw, nx, ny)}
        if fields:
            shapes.update({"U": (nw, nx, ny, nz + 6), "kappa": (nw, nx, ny, nz), "V": (nw, nx, ny, nz)})
        given = out or {}
        out = {}
        for k, shp in shapes.items():
            if k in given:
                _need_host(k, given[k], int(np.prod(shp)))
                out[k] = given[k]
            else:
                out[k] = np.empty(shp)
        self._check(self.lib.oco_server_fetch(self.h, int(jid), _ptr(out["Vtop"]), _ptr(out["Vbot"]),
                                              _ptr(out.get("U")), _ptr(out.get("kappa")), _ptr(out.get("V"))))
        del self._jobs[jid]
        return out

    def close(self):
        if self.h:
            self.lib.oco_server_destroy(self.h)
            self.h = ctypes.c_void_p()
            self._jobs.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
