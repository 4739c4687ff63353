"""Python API of the B200 structure-factor path, on torch device tensors.

    mol = Molecule(Z, pos)                     # host arrays; atoms go to the GPU once
    qs = QSet.from_detector(256, 256, ...)     # Ewald q of every pixel, FP64 on the GPU
    F, I = forward(mol, qs)                    # complex64 F and |F|^2, CUDA tensors
    out = detector_chain(params, I)            # Thomson ... ADC, CUDA tensors

PyTorch provides device memory and streams only; every kernel is the
library's own (spsim_b200/csrc).  Arguments and errors follow the native ABI
in include/spsim_b200.h: a non-zero status raises SpsimError.
"""
import ctypes
from ctypes import byref, c_double, c_int, c_int64, c_void_p

import numpy as np
import torch

from . import _native
from ._native import PRECISIONS, ChainOutputs, ChainParams, check, lib

__all__ = [
    "Molecule", "QSet", "forward", "forward_batch", "adjoint", "detector_chain", "chain_params",
    "hkl_for_detector", "synchronize", "forward_spectrum", "timing", "autotune", "set_variant", "last_forward_stats",
    "last_variant", "last_phase_word", "last_pair_narrow", "kernel_name", "autotune_batch", "clear_tuning",
    "forward_nufft", "forward_nufft_batch", "last_nufft_grid",
]


def _prec(p):
    if isinstance(p, str):
        return PRECISIONS[p]
    return int(p)


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return c_void_p(s.cuda_stream)


def _dev(t):
    return c_void_p(t.data_ptr()) if t is not None else None


def _ensure_device(device=None):
    idx = torch.cuda.current_device() if device is None else torch.device(device).index or 0
    _native.use_device(idx)
    return idx


def _host(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


class Molecule:
    """Device-resident atoms of one molecule (element-sorted, centred, split)."""

    def __init__(self, Z, pos, occ=None, bfac=None, delta_atoms=False, beam=None, device=None):
        self.device = _ensure_device(device)
        Z = _host(Z, np.int32).reshape(-1)
        pos = np.asarray(pos)
        pos64 = pos.dtype == np.float64
        pos = _host(pos, np.float64 if pos64 else np.float32).reshape(-1, 3)
        if pos.shape[0] != Z.shape[0]:
            raise ValueError("Z and pos disagree on the number of atoms")
        occ_a = _host(occ, np.float32).reshape(-1) if occ is not None else None
        b_a = _host(bfac, np.float32).reshape(-1) if bfac is not None else None
        beam_a = _host(beam, np.float32).reshape(3) if beam is not None else None
        h = c_void_p()
        fn = lib().spsim_b200_molecule_create_f64 if pos64 else lib().spsim_b200_molecule_create
        check(fn(int(Z.shape[0]), Z.ctypes.data_as(c_void_p), pos.ctypes.data_as(c_void_p),
                 occ_a.ctypes.data_as(c_void_p) if occ_a is not None else None,
                 b_a.ctypes.data_as(c_void_p) if b_a is not None else None, int(bool(delta_atoms)),
                 beam_a.ctypes.data_as(c_void_p) if beam_a is not None else None, byref(h)))
        self.handle = h
        self.natoms = int(Z.shape[0])
        self.n_kept = int(np.count_nonzero(Z))
        self.per_atom_b = bfac is not None

    def update_device(self, pos, occ=None, bfac=None, stream=None):
        """Rewrite positions (N,3 CUDA tensor, float32/64), occupancies and B factors in place."""
        _native.use_device(self.device)
        pos = pos.contiguous()
        occ = occ.contiguous().float() if occ is not None else None
        bfac = bfac.contiguous().float() if bfac is not None else None
        check(lib().spsim_b200_molecule_update_device(self.handle, _dev(pos), int(pos.dtype == torch.float64),
                                                      _dev(occ), _dev(bfac), _stream_ptr(stream)))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                lib().spsim_b200_molecule_destroy(h)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self.handle = None


class QSet:
    """Device-resident scattering vectors of one detector (1/m)."""

    def __init__(self, handle, npix, device):
        self.handle = handle
        self.npix = npix
        self.device = device

    @classmethod
    def from_list(cls, hkl, device=None):
        """From the reference's float HKL list: numpy (host) or CUDA tensor, shape (npix, 3)."""
        dev = _ensure_device(device)
        h = c_void_p()
        if isinstance(hkl, torch.Tensor) and hkl.is_cuda:
            t = hkl.reshape(-1, 3).contiguous().float()
            check(lib().spsim_b200_qset_from_list(t.shape[0], _dev(t), _native.MEM_DEVICE, byref(h)))
            n = t.shape[0]
        else:
            a = _host(hkl, np.float32).reshape(-1, 3)
            check(lib().spsim_b200_qset_from_list(a.shape[0], a.ctypes.data_as(c_void_p), _native.MEM_HOST, byref(h)))
            n = a.shape[0]
        return cls(h, int(n), dev)

    @classmethod
    def from_detector(cls, nx, ny, width, height, distance, wavelength, center_x=0.0, center_y=0.0, spherical=False,
                      device=None):
        """Ewald-sphere q of a flat (or spherical) detector, FP64 on the device."""
        dev = _ensure_device(device)
        h = c_void_p()
        check(lib().spsim_b200_qset_from_detector(int(nx), int(ny), float(width), float(height), float(distance),
                                                  float(center_x), float(center_y), float(wavelength),
                                                  int(bool(spherical)), byref(h)))
        return cls(h, int(nx) * int(ny), dev)

    def q(self):
        """The q vectors as a (npix, 3) float32 numpy array."""
        out = np.empty((self.npix, 3), np.float32)
        check(lib().spsim_b200_qset_copy_q(self.handle, out.ctypes.data_as(c_void_p)))
        return out

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                lib().spsim_b200_qset_destroy(h)
            except Exception:  # noqa: BLE001
                pass
            self.handle = None


def _rot_array(rot, n):
    if rot is None:
        return None
    r = np.ascontiguousarray(np.asarray(rot, np.float64).reshape(n, 9))
    return r


def forward(mol, qs, rot=None, B=0.0, precision="f32", F=None, I=None, want_F=True, want_I=True, stream=None):
    """One pattern.  Returns (F, I): F complex64 (npix,), I float32 (npix,) CUDA tensors."""
    _native.use_device(mol.device)
    dev = torch.device("cuda", mol.device)
    if want_F and F is None:
        F = torch.empty(qs.npix, dtype=torch.complex64, device=dev)
    if want_I and I is None:
        I = torch.empty(qs.npix, dtype=torch.float32, device=dev)
    r = _rot_array(rot, 1)
    check(lib().spsim_b200_forward(mol.handle, qs.handle, r.ctypes.data_as(c_void_p) if r is not None else None,
                                   float(B), _prec(precision), _dev(F) if want_F else None,
                                   _dev(I) if want_I else None, _stream_ptr(stream)))
    return (F if want_F else None), (I if want_I else None)


def forward_nufft(mol, qs, rot=None, B=0.0, eps=1e-8, F=None, I=None, want_F=True, want_I=True, stream=None):
    """The structure factor of forward() by a type-3 non-uniform FFT per
    element (FP64 grids and hand-written pruned FFT passes), for large molecules: relative L2 error of F
    about eps against the exact sum.  Replaces spsim's NNFFT path
    (src/diffraction.c:528-675).  Returns (F, I) like forward()."""
    _native.use_device(mol.device)
    dev = torch.device("cuda", mol.device)
    if want_F and F is None:
        F = torch.empty(qs.npix, dtype=torch.complex64, device=dev)
    if want_I and I is None:
        I = torch.empty(qs.npix, dtype=torch.float32, device=dev)
    r = _rot_array(rot, 1)
    check(lib().spsim_b200_forward_nufft(mol.handle, qs.handle, r.ctypes.data_as(c_void_p) if r is not None else None,
                                         float(B), float(eps), _dev(F) if want_F else None,
                                         _dev(I) if want_I else None, _stream_ptr(stream)))
    return (F if want_F else None), (I if want_I else None)


def forward_nufft_batch(mol, qs, rots, B=0.0, eps=1e-8, F=None, I=None, want_F=True, want_I=True, stream=None):
    """Many orientations of one molecule by the NUFFT: the grid is sized for
    every rotation, the atoms are spread and transformed once, each pattern is
    one interpolation pass.  rots: (npat, 3, 3).  Returns (F, I) of shape
    (npat, npix)."""
    _native.use_device(mol.device)
    dev = torch.device("cuda", mol.device)
    r = np.ascontiguousarray(np.asarray(rots, np.float64).reshape(-1, 9))
    npat = r.shape[0]
    if want_F and F is None:
        F = torch.empty(npat, qs.npix, dtype=torch.complex64, device=dev)
    if want_I and I is None:
        I = torch.empty(npat, qs.npix, dtype=torch.float32, device=dev)
    check(lib().spsim_b200_forward_nufft_batch(mol.handle, qs.handle, int(npat), r.ctypes.data_as(c_void_p),
                                               float(B), float(eps), _dev(F) if want_F else None,
                                               _dev(I) if want_I else None, _stream_ptr(stream)))
    return (F if want_F else None), (I if want_I else None)


def set_nufft_interp(mode):
    """NUFFT interpolation path: 0 (default) the shared-memory tile path for
    detector q sets, 1 per-pixel stencil reads everywhere (same bits)."""
    check(lib().spsim_b200_set_nufft_interp(int(mode)))


def last_nufft_grid():
    """(spreading width, interpolation width, (n2x, n2y, n2z)) of the last NUFFT forward on this thread."""
    a, b = c_int(0), c_int(0)
    n = (c_int * 3)()
    check(lib().spsim_b200_last_nufft_grid(byref(a), byref(b), n))
    return a.value, b.value, tuple(n)


def forward_spectrum(mol, qs, wavelength, bandwidth, samples=5, rot=None, B=0.0, precision="f32", F=None, I=None,
                     want_F=True, want_I=True, stream=None):
    """Polychromatic pattern with spsim's spectrum-kernel semantics
    (src/diffraction.cu:415-476): the amplitude averaged over `samples`
    wavelengths across the relative bandwidth, Gaussian-weighted, all samples
    in one batched launch.  Returns (F, I) like forward()."""
    _native.use_device(mol.device)
    dev = torch.device("cuda", mol.device)
    if want_F and F is None:
        F = torch.empty(qs.npix, dtype=torch.complex64, device=dev)
    if want_I and I is None:
        I = torch.empty(qs.npix, dtype=torch.float32, device=dev)
    r = _rot_array(rot, 1)
    check(lib().spsim_b200_forward_spectrum(mol.handle, qs.handle,
                                            r.ctypes.data_as(c_void_p) if r is not None else None, float(B),
                                            _prec(precision), float(wavelength), float(bandwidth), int(samples),
                                            _dev(F) if want_F else None, _dev(I) if want_I else None,
                                            _stream_ptr(stream)))
    return (F if want_F else None), (I if want_I else None)


def forward_batch(mols, qsets, rots=None, B=0.0, precision="f32", F=None, I=None, want_F=True, want_I=True,
                  stream=None):
    """Many patterns in one persistent launch (graph-replayed when repeated).

    mols / qsets: sequences of equal length (or a single object broadcast);
    rots: (npat, 3, 3) FP64 rotations or None.  Returns lists of tensors."""
    if rots is not None:
        npat = len(rots)
    else:
        npat = len(mols) if isinstance(mols, (list, tuple)) else len(qsets)
    mols = list(mols) if isinstance(mols, (list, tuple)) else [mols] * npat
    qsets = list(qsets) if isinstance(qsets, (list, tuple)) else [qsets] * npat
    if len(mols) != npat or len(qsets) != npat:
        raise ValueError("molecules, q sets and rotations disagree on the number of patterns")
    _native.use_device(mols[0].device)
    dev = torch.device("cuda", mols[0].device)
    if want_F and F is None:
        F = [torch.empty(q.npix, dtype=torch.complex64, device=dev) for q in qsets]
    if want_I and I is None:
        I = [torch.empty(q.npix, dtype=torch.float32, device=dev) for q in qsets]
    MA = c_void_p * npat
    mh = MA(*[m.handle.value for m in mols])
    qh = MA(*[q.handle.value for q in qsets])
    fh = MA(*[t.data_ptr() for t in F]) if want_F else None
    ih = MA(*[t.data_ptr() for t in I]) if want_I else None
    r = _rot_array(rots, npat)
    check(lib().spsim_b200_forward_batch(npat, ctypes.cast(mh, c_void_p), ctypes.cast(qh, c_void_p),
                                         r.ctypes.data_as(c_void_p) if r is not None else None, float(B),
                                         _prec(precision), ctypes.cast(fh, c_void_p) if fh else None,
                                         ctypes.cast(ih, c_void_p) if ih else None, _stream_ptr(stream)))
    return (F if want_F else None), (I if want_I else None)


def adjoint(mol, qs, F, G, rots=None, B=0.0, precision="f32", want_occ=True, want_b=None, stream=None):
    """dL/dpos (natoms,3), dL/docc (natoms,), dL/dB (natoms,) as float64 CUDA tensors.

    F: complex64 (npat*npix) forward amplitudes; G: float32 dL/dI, same shape."""
    _native.use_device(mol.device)
    dev = torch.device("cuda", mol.device)
    npat = 1 if rots is None else len(rots)
    F = F.reshape(-1).contiguous()
    G = G.reshape(-1).contiguous().float()
    if F.numel() != npat * qs.npix or G.numel() != npat * qs.npix:
        raise ValueError("F and G must hold npat * npix values")
    want_b = mol.per_atom_b if want_b is None else want_b
    dpos = torch.empty(mol.natoms, 3, dtype=torch.float64, device=dev)
    docc = torch.empty(mol.natoms, dtype=torch.float64, device=dev) if want_occ else None
    dB = torch.empty(mol.natoms, dtype=torch.float64, device=dev) if want_b else None
    r = _rot_array(rots, npat)
    check(lib().spsim_b200_adjoint(mol.handle, qs.handle, npat, r.ctypes.data_as(c_void_p) if r is not None else None,
                                   float(B), _prec(precision), _dev(F), _dev(G), _dev(dpos), _dev(docc), _dev(dB),
                                   _stream_ptr(stream)))
    return dpos, docc, dB


CHAIN_FIELDS = [f for f, _ in ChainParams._fields_]


def chain_params(**kw):
    """spsim_b200_chain_params from keyword arguments (unset fields: 0, binning 1, nz 1)."""
    p = ChainParams()
    p.nz = 1
    p.binning_x = p.binning_y = p.binning_z = 1
    for k, v in kw.items():
        if k not in CHAIN_FIELDS:
            raise KeyError("unknown chain parameter %r" % k)
        setattr(p, k, v)
    return p


CHAIN_OUTPUTS = ["thomson_correction", "solid_angle", "photons_per_pixel", "photon_count", "electrons_per_pixel",
                 "real_output", "noiseless_output"]


def detector_chain(params, I, outputs=CHAIN_OUTPUTS, stream=None):
    """Fused detector chain on intensities I (CUDA float32, nx*ny*nz).  Returns a dict of tensors."""
    dev = I.device if I is not None else torch.device("cuda", torch.cuda.current_device())
    _native.use_device(dev.index or 0)
    n = params.nx * params.ny * params.nz
    nb = (params.nx // params.binning_x) * (params.ny // params.binning_y) * (params.nz // params.binning_z)
    res = {}
    o = ChainOutputs()
    for name in outputs:
        t = torch.empty(nb if name in ("real_output", "noiseless_output") else n, dtype=torch.float32, device=dev)
        res[name] = t
        setattr(o, name, t.data_ptr())
    Ic = I.contiguous() if I is not None else None  # held until the launch is enqueued
    check(lib().spsim_b200_detector_chain(byref(params), _dev(Ic), byref(o), _stream_ptr(stream)))
    return res


def hkl_for_detector(nx, ny, width, height, distance, wavelength, center_x=0.0, center_y=0.0, spherical=False,
                     stream=None):
    """The reference HKL list (float32, (nx*ny, 3)) as a CUDA tensor."""
    _ensure_device()
    out = torch.empty(int(nx) * int(ny), 3, dtype=torch.float32, device="cuda")
    check(lib().spsim_b200_hkl_for_detector(int(nx), int(ny), float(width), float(height), float(distance),
                                            float(center_x), float(center_y), float(wavelength),
                                            int(bool(spherical)), _dev(out), _stream_ptr(stream)))
    return out


def poisson(lam, seed, pattern_index=0, stream=None):
    """Philox Poisson deviates of a CUDA float32 tensor of means."""
    _native.use_device(lam.device.index or 0)
    lam = lam.contiguous().float()
    out = torch.empty_like(lam)
    check(lib().spsim_b200_poisson(lam.numel(), _dev(lam), int(seed), int(pattern_index), _dev(out),
                                   _stream_ptr(stream)))
    return out


def synchronize(stream=None):
    check(lib().spsim_b200_synchronize(_stream_ptr(stream)))


class timing:
    """Context manager: per-launch CUDA-event timing of structure-factor kernels.

        with timing() as t:
            forward(...)
        t.ms  # list of kernel durations (ms)
    """

    def __enter__(self):
        check(lib().spsim_b200_timing_enable(1))
        self.ms = []
        return self

    def read(self, cap=100000):
        buf = (c_double * cap)()
        n = c_int(0)
        check(lib().spsim_b200_timing_read(buf, cap, byref(n)))
        self.ms.extend(buf[i] for i in range(n.value))
        return self.ms

    def __exit__(self, *exc):
        self.read()
        check(lib().spsim_b200_timing_enable(0))
        return False


def last_forward_stats():
    t = c_double(0)
    ms = c_double(0)
    check(lib().spsim_b200_last_forward_stats(byref(t), byref(ms)))
    return t.value, ms.value


FORMS = {0: "compensated FP32, one pixel per lane", 1: "compensated FP32, pixel pairs (f32x2)",
         2: "FP64 phase, FP32 sin/cos on pixel pairs (f32x2)",
         3: "FP64 phase on the first pixel of neighbour pairs, FP32 step to the second",
         4: "FP64 phase on the second pixel of neighbour quads, FP32 steps to the other three"}
KERNELS = {-1: "sf_f64_kernel", 0: "sf_f32_kernel", 1: "sf_f32x2_kernel", 2: "sf_dphase_kernel", 3: "sf_dpair_kernel",
           4: "sf_dquad_kernel"}


def last_variant():
    """(threads, pixels_per_thread, form) of the last forward on this thread; form -1 = plain FP64."""
    t, p, f = c_int(0), c_int(0), c_int(0)
    check(lib().spsim_b200_last_variant(byref(t), byref(p), byref(f)))
    return t.value, p.value, f.value


def last_phase_word():
    """True when the last forward on this thread (forms 2, 3, 4) took its phases
    from the fixed-point phase word rather than FP64 rounding."""
    on = c_int(0)
    check(lib().spsim_b200_last_phase_word(byref(on)))
    return bool(on.value)


def last_pair_narrow():
    """True when the last forward on this thread ran the neighbour-pair form
    (3) with every pair's step within 0.07 cycle, or the neighbour-quad form
    (4) with every one-pixel step within 0.07 cycle, those pixels on the
    shorter NARROW sin/cos polynomial."""
    on = c_int(0)
    check(lib().spsim_b200_last_pair_narrow(byref(on)))
    return bool(on.value)


def kernel_name():
    """Name of the structure-factor kernel the last forward on this thread ran."""
    return KERNELS[last_variant()[2]]


def set_variant(threads=-1, pixels_per_thread=-1, form=4):
    """Force an FP32 kernel variant: threads per CTA, pixels per thread and the
    kernel form (FORMS); threads < 0 returns to automatic choice."""
    check(lib().spsim_b200_set_variant(int(threads), int(pixels_per_thread), int(form)))


def autotune(mol, qs, precision="f32", stream=None):
    """Time every compiled FP32 kernel variant on this workload; returns (threads, pixels_per_thread, form)."""
    _native.use_device(mol.device)
    bt, bp, bk = c_int(0), c_int(0), c_int(0)
    check(lib().spsim_b200_autotune(mol.handle, qs.handle, _prec(precision), _stream_ptr(stream), byref(bt),
                                    byref(bp), byref(bk)))
    return bt.value, bp.value, bk.value


def autotune_batch(mols, qsets, rots=None, precision="f32", stream=None):
    """Time every compiled FP32 kernel variant on one batched forward of these
    patterns (arguments as forward_batch) and keep the fastest for batches of
    this size; returns (threads, pixels_per_thread, form)."""
    if rots is not None:
        npat = len(rots)
    else:
        npat = len(mols) if isinstance(mols, (list, tuple)) else len(qsets)
    mols = list(mols) if isinstance(mols, (list, tuple)) else [mols] * npat
    qsets = list(qsets) if isinstance(qsets, (list, tuple)) else [qsets] * npat
    if len(mols) != npat or len(qsets) != npat:
        raise ValueError("molecules, q sets and rotations disagree on the number of patterns")
    _native.use_device(mols[0].device)
    MA = c_void_p * npat
    mh = MA(*[m.handle.value for m in mols])
    qh = MA(*[q.handle.value for q in qsets])
    r = _rot_array(rots, npat)
    bt, bp, bk = c_int(0), c_int(0), c_int(0)
    check(lib().spsim_b200_autotune_batch(npat, ctypes.cast(mh, c_void_p), ctypes.cast(qh, c_void_p),
                                          r.ctypes.data_as(c_void_p) if r is not None else None, _prec(precision),
                                          _stream_ptr(stream), byref(bt), byref(bp), byref(bk)))
    return bt.value, bp.value, bk.value


def clear_tuning():
    """Forget every autotuned choice: later forwards use the untuned defaults."""
    check(lib().spsim_b200_clear_tuning())


def npix_of(qs):
    n = c_int64(0)
    check(lib().spsim_b200_qset_npix(qs.handle, byref(n)))
    return n.value
