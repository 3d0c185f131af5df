"""`Ssimulacra2` and `Ssim2Batch`: the reference's host API over the C ABI.

Reference: crates/ssimulacra2-cuda/src/lib.rs (Ssimulacra2::new :80,
compute :421, compute_sync :409, get_score :427, compute_srgb_sync :391,
compute_from_cpu_srgb_sync :329, set_reference_linear :440,
compute_with_reference_linear :556, clear_reference :595, has_reference :600,
mem_usage :207) and crates/ssim2-gpu/src/pipeline_batch.rs (Ssim2Batch).

Images on the device are torch CUDA tensors:
  linear f32   (H, W, 3) float32, rows may be padded (stride(0) >= 3W)
  sRGB8        (H, W, 3) uint8
  NV12         y (H, W) uint8 and uv (H/2, W) uint8, same row stride
  RGB16        (H, W, 3) uint16
or `(pointer, pitch_bytes)` tuples.  Host images are numpy arrays of the
same shapes.
"""
import collections
import ctypes

import numpy as np

from . import capi
from .capi import lib, check, NUM_STATS


def _stream_ptr(stream):
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        except ImportError:
            pass
        return None
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


def _dev(img, elem_bytes):
    """(pointer, pitch in bytes) of a device image."""
    if isinstance(img, tuple):
        return ctypes.c_void_p(img[0]), img[1]
    if not img.is_cuda:
        raise capi.S2Error(capi.S2_ERR_INVALID_ARG, "expected a CUDA tensor")
    if img.stride(-1) != 1 or (img.dim() == 3 and img.stride(1) != img.shape[2]):
        raise capi.S2Error(capi.S2_ERR_INVALID_ARG, "rows must be packed samples")
    return ctypes.c_void_p(img.data_ptr()), img.stride(0) * elem_bytes


def _host_ptr(img, elem_bytes):
    """(pointer, pitch in bytes) of a host image: a CPU torch tensor (pinned
    for asynchronous uploads) or a numpy array with packed rows."""
    if isinstance(img, tuple):
        return ctypes.c_void_p(img[0]), img[1]
    if isinstance(img, np.ndarray):
        if img.strides[-1] != img.itemsize or (img.ndim == 3 and img.strides[1] != img.shape[2] * img.itemsize):
            raise capi.S2Error(capi.S2_ERR_INVALID_ARG, "rows must be packed samples")
        return ctypes.c_void_p(img.ctypes.data), img.strides[0]
    if img.is_cuda:
        raise capi.S2Error(capi.S2_ERR_INVALID_ARG, "expected a host (CPU) tensor")
    if img.stride(-1) != 1 or (img.dim() == 3 and img.stride(1) != img.shape[2]):
        raise capi.S2Error(capi.S2_ERR_INVALID_ARG, "rows must be packed samples")
    return ctypes.c_void_p(img.data_ptr()), img.stride(0) * elem_bytes


def _host(img):
    a = np.ascontiguousarray(img)
    return a.ctypes.data_as(ctypes.c_void_p), a.strides[0], a


class Ssimulacra2:
    """One (reference, distorted) size; see crates/ssimulacra2-cuda/src/lib.rs:27-77.

    Unlike the reference, the instance is not bound to input buffers: every
    compute call names them.  `Ssimulacra2.new(ref, dis)` keeps the reference's
    binding style (`compute()` then re-reads those two tensors)."""

    def __init__(self, width, height, *, device=0, storage="f32", scale_rule="cpu", strip_rows=0,
                 hbm_budget=0, blur="fir"):
        self.width, self.height = int(width), int(height)
        cfg = capi.make_config(device=device, storage=storage, scale_rule=scale_rule,
                               strip_rows=strip_rows, hbm_budget=hbm_budget, blur=blur)
        h = ctypes.c_void_p()
        check(lib.s2_create(ctypes.byref(cfg), self.width, self.height, ctypes.byref(h)), "Ssimulacra2::new")
        self._h = h
        self._bound = None
        self._keep = None

    @classmethod
    def new(cls, src_ref_linear, src_dis_linear, stream=None, **kw):
        """Ssimulacra2::new (lib.rs:80): size from the images, bound to them."""
        if tuple(src_ref_linear.shape) != tuple(src_dis_linear.shape):
            raise capi.DimensionMismatch(capi.S2_ERR_DIM_MISMATCH, "Ssimulacra2::new")
        h, w = src_ref_linear.shape[:2]
        s = cls(w, h, **kw)
        s._bound = (src_ref_linear, src_dis_linear)
        return s

    def error_maps(self, scale, stream=None):
        """The last compute's error maps at `scale` as a (3, 3, h_s, w_s) float32
        CUDA tensor: [channel X, Y, B][ssim, artifact, detail]."""
        import torch
        w, h = self.width, self.height
        for _ in range(scale):
            w, h = (w + 1) // 2, (h + 1) // 2
        out = torch.empty((3, 3, h, w), dtype=torch.float32, device="cuda")
        check(lib.s2_error_maps(self._h, int(scale), ctypes.c_void_p(out.data_ptr()), w * 4, _stream_ptr(stream)),
              "error_maps")
        return out

    def set_graphs(self, enable=True):
        """Replay computes of a seen shape as CUDA graphs (default on)."""
        check(lib.s2_set_graphs(self._h, 1 if enable else 0), "set_graphs")

    def close(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.s2_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_metrics(self, metrics):
        """Metrics of later computes: 'ssimulacra2', 'dssim' or both."""
        check(lib.s2_set_metrics(self._h, capi.metrics_mask(metrics)), "set_metrics")

    def get_dssim(self):
        """(dssim, per-scale scores[5]) of the last compute (DSSIM scored)."""
        v = ctypes.c_double()
        sc = np.zeros(5)
        check(lib.s2_get_dssim(self._h, ctypes.byref(v), sc.ctypes.data_as(capi.D)), "get_dssim")
        return v.value, sc

    # -- reference API ------------------------------------------------------
    def mem_usage(self):
        n = ctypes.c_size_t()
        check(lib.s2_mem_usage(self._h, ctypes.byref(n)), "mem_usage")
        return n.value

    def compute(self, stream=None):
        """Ssimulacra2::compute (lib.rs:421): enqueue on the bound images."""
        if self._bound is None:
            raise capi.S2Error(capi.S2_ERR_INVALID_ARG, "compute: no bound images (use compute_linear)")
        self.compute_linear(self._bound[0], self._bound[1], stream)

    def compute_sync(self, stream=None):
        """Ssimulacra2::compute_sync (lib.rs:409)."""
        self.compute(stream)
        return self.get_score()

    def get_score(self):
        """Ssimulacra2::get_score (lib.rs:427); idempotent."""
        return self.get_result()[0]

    def get_result(self):
        """(score, stats[108], sums[108]) of the last compute."""
        sc = ctypes.c_double()
        st = np.zeros(NUM_STATS)
        su = np.zeros(NUM_STATS)
        check(lib.s2_get_result(self._h, ctypes.byref(sc), st.ctypes.data_as(capi.D),
                                su.ctypes.data_as(capi.D)), "get_score")
        return sc.value, st, su

    def compute_linear(self, ref, dis, stream=None):
        rp, rpitch = _dev(ref, 4)
        dp, dpitch = _dev(dis, 4)
        self._keep = (ref, dis)
        check(lib.s2_compute_linear_f32(self._h, rp, rpitch, dp, dpitch, _stream_ptr(stream)), "compute")

    def compute_srgb(self, src_ref, src_dis, stream=None):
        rp, rpitch = _dev(src_ref, 1)
        dp, dpitch = _dev(src_dis, 1)
        self._keep = (src_ref, src_dis)
        check(lib.s2_compute_srgb8(self._h, rp, rpitch, dp, dpitch, 0, _stream_ptr(stream)), "compute_srgb")

    def compute_srgb_sync(self, src_ref, src_dis, stream=None):
        """compute_srgb_sync (lib.rs:391): device sRGB8 pair -> score."""
        self.compute_srgb(src_ref, src_dis, stream)
        return self.get_score()

    def compute_from_cpu_srgb_sync(self, ref_bytes, dis_bytes, stream=None):
        """compute_from_cpu_srgb_sync (lib.rs:329): host sRGB8 (H, W, 3) pair."""
        rp, rpitch, ra = _host(ref_bytes)
        dp, dpitch, da = _host(dis_bytes)
        self._check_host(ra, 3)
        self._check_host(da, 3)
        check(lib.s2_compute_srgb8(self._h, rp, rpitch, dp, dpitch, 1, _stream_ptr(stream)), "compute_from_cpu")
        return self.get_score()

    def _yuv420(self, fn, es, ref_y, ref_uv, dis_y, dis_uv, matrix, range_, stream, on_host):
        if on_host:
            ry, rpitch, a1 = _host(ref_y)
            ru, _, a2 = _host(ref_uv)
            dy, dpitch, a3 = _host(dis_y)
            du, _, a4 = _host(dis_uv)
            self._keep = (a1, a2, a3, a4)
        else:
            ry, rpitch = _dev(ref_y, es)
            ru, _ = _dev(ref_uv, es)
            dy, dpitch = _dev(dis_y, es)
            du, _ = _dev(dis_uv, es)
            self._keep = (ref_y, ref_uv, dis_y, dis_uv)
        check(fn(self._h, ry, ru, rpitch, dy, du, dpitch, capi.MATRIX[matrix], capi.RANGE[range_], int(on_host),
                 _stream_ptr(stream)), fn.__name__)

    def compute_nv12(self, ref_y, ref_uv, dis_y, dis_uv, stream=None, on_host=False, matrix="bt709",
                     range="limited"):
        """8-bit 4:2:0 biplanar pair: Y (H, W) and interleaved CbCr (H/2, W) planes."""
        self._yuv420(lib.s2_compute_nv12, 1, ref_y, ref_uv, dis_y, dis_uv, matrix, range, stream, on_host)

    def compute_p016(self, ref_y, ref_uv, dis_y, dis_uv, stream=None, on_host=False, matrix="bt709",
                     range="limited"):
        """16-bit 4:2:0 biplanar pair (P016; P010/P012 data left-aligned): uint16 / int16 planes."""
        self._yuv420(lib.s2_compute_p016, 2, ref_y, ref_uv, dis_y, dis_uv, matrix, range, stream, on_host)

    def compute_rgb16(self, ref, dis, bits=10, stream=None, on_host=False):
        if on_host:
            rp, rpitch, a1 = _host(ref)
            dp, dpitch, a2 = _host(dis)
            self._keep = (a1, a2)
        else:
            rp, rpitch = _dev(ref, 2)
            dp, dpitch = _dev(dis, 2)
            self._keep = (ref, dis)
        check(lib.s2_compute_rgb16(self._h, rp, rpitch, dp, dpitch, bits, int(on_host), _stream_ptr(stream)),
              "compute_rgb16")

    # -- cached reference ----------------------------------------------------
    def set_reference_linear(self, src_ref_linear, stream=None):
        """set_reference_linear (lib.rs:440)."""
        rp, rpitch = _dev(src_ref_linear, 4)
        check(lib.s2_set_reference_linear_f32(self._h, rp, rpitch, _stream_ptr(stream)), "set_reference_linear")

    def set_reference_srgb(self, ref, stream=None, on_host=False):
        if on_host:
            rp, rpitch, a = _host(ref)
            self._check_host(a, 3)
        else:
            rp, rpitch = _dev(ref, 1)
        check(lib.s2_set_reference_srgb8(self._h, rp, rpitch, int(on_host), _stream_ptr(stream)), "set_reference")

    def compute_with_reference_linear(self, src_dis_linear, stream=None):
        """compute_with_reference_linear (lib.rs:556); raises NoCachedReference
        where the reference panics."""
        dp, dpitch = _dev(src_dis_linear, 4)
        self._keep = (src_dis_linear,)
        check(lib.s2_compute_with_reference_linear_f32(self._h, dp, dpitch, _stream_ptr(stream)),
              "compute_with_reference_linear")
        return self.get_score()

    def compute_with_reference_srgb(self, dis, stream=None, on_host=False):
        if on_host:
            dp, dpitch, a = _host(dis)
            self._check_host(a, 3)
        else:
            dp, dpitch = _dev(dis, 1)
        self._keep = (dis,)
        check(lib.s2_compute_with_reference_srgb8(self._h, dp, dpitch, int(on_host), _stream_ptr(stream)),
              "compute_with_reference")
        return self.get_score()

    def clear_reference(self):
        check(lib.s2_clear_reference(self._h), "clear_reference")

    def has_reference(self):
        return bool(lib.s2_has_reference(self._h))

    def _check_host(self, a, ch):
        if a.shape[0] != self.height or a.shape[1] != self.width or (a.ndim == 3 and a.shape[2] != ch):
            raise capi.DimensionMismatch(capi.S2_ERR_DIM_MISMATCH, "host image shape")


class PairDesc:
    """One pair of a batch: device tensors of any supported format (host arrays
    for `Ssim2Batch.submit_host`)."""

    def __init__(self, ref, dis, fmt="srgb8", ref_uv=None, dis_uv=None, bits=10, matrix="bt709", range="limited"):
        self.ref, self.dis, self.fmt, self.ref_uv, self.dis_uv, self.bits = ref, dis, fmt, ref_uv, dis_uv, bits
        self.matrix, self.range = matrix, range

    def to_c(self, host=False):
        d = capi.PairDescC()
        eb = {"linear_f32": 4, "srgb8": 1, "nv12": 1, "rgb16": 2, "p016": 2}[self.fmt]
        ptr = _host_ptr if host else _dev
        rp, rpitch = ptr(self.ref, eb)
        dp, dpitch = ptr(self.dis, eb)
        d.height, d.width = self.ref.shape[0], self.ref.shape[1]
        d.format = capi.FMT[self.fmt]
        d.bits = self.bits
        d.ref, d.dis = rp.value, dp.value
        d.ref_pitch, d.dis_pitch = rpitch, dpitch
        if self.fmt in ("nv12", "p016"):
            d.ref_uv = ptr(self.ref_uv, eb)[0].value
            d.dis_uv = ptr(self.dis_uv, eb)[0].value
            d.matrix = capi.MATRIX[self.matrix]
            d.range = capi.RANGE[self.range]
        return d


class Ssim2Batch:
    """Many pairs of any sizes per submission (ssim2-gpu pipeline_batch.rs:120-382,
    widened to mixed sizes and formats)."""

    def __init__(self, max_pairs, max_pixels, *, device=0, storage="f32", scale_rule="cpu", strip_rows=0,
                 hbm_budget=0, blur="fir"):
        cfg = capi.make_config(device=device, storage=storage, scale_rule=scale_rule, strip_rows=strip_rows,
                               hbm_budget=hbm_budget, blur=blur)
        h = ctypes.c_void_p()
        check(lib.s2_batch_create(ctypes.byref(cfg), max_pairs, max_pixels, ctypes.byref(h)), "Ssim2Batch::new")
        self._h = h
        self.max_pairs = max_pairs
        # submissions whose results were not read, oldest first: (slot, n,
        # pairs kept alive) -- the same slot rule as s2_batch (two slots;
        # device submissions use slot 0, host ones a slot without pending
        # results)
        self._unread = collections.deque()
        self._last = (0, 0, None)

    def _take_slot(self, host):
        pending = [u[0] for u in self._unread]
        k = 0
        if host and 0 in pending:
            k = self._unread[0][0] if 1 in pending else 1
        self._unread = collections.deque(u for u in self._unread if u[0] != k)
        return k

    def close(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.s2_batch_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def submit(self, pairs, stream=None):
        arr = (capi.PairDescC * max(len(pairs), 1))()
        for i, p in enumerate(pairs):
            arr[i] = p.to_c()
        k = self._take_slot(False)
        check(lib.s2_batch_submit(self._h, arr, len(pairs), _stream_ptr(stream)), "compute_batch")
        self._last = (k, len(pairs), pairs)
        self._unread.append(self._last)

    def set_graphs(self, enable=True):
        """Replay submissions of a seen shape as CUDA graphs (default on)."""
        check(lib.s2_batch_set_graphs(self._h, 1 if enable else 0), "set_graphs")

    def set_metrics(self, metrics):
        """Metrics of later submissions: 'ssimulacra2', 'dssim' or both (one
        prep pass feeds both); results then carry the DSSIM value and its
        per-scale scores (NaN when DSSIM is not scored)."""
        check(lib.s2_batch_set_metrics(self._h, capi.metrics_mask(metrics)), "set_metrics")

    def submit_host(self, pairs, stream=None):
        """Pairs whose planes are in host memory (CPU tensors, pinned for
        overlap, or numpy arrays): uploaded in groups that overlap the compute
        of earlier groups.  Keep the arrays alive and unchanged until
        `results()` returns.  A second host submission may be made before
        reading the first one's results: its uploads and preps then overlap
        the first one's tile pass (results are read oldest first)."""
        arr = (capi.PairDescC * max(len(pairs), 1))()
        for i, p in enumerate(pairs):
            arr[i] = p.to_c(host=True)
        k = self._take_slot(True)
        check(lib.s2_batch_submit_host(self._h, arr, len(pairs), _stream_ptr(stream)), "compute_batch_host")
        self._last = (k, len(pairs), pairs)
        self._unread.append(self._last)

    def results(self):
        """Results of the oldest submission not read yet (else the last one)."""
        _, n, _ = self._unread.popleft() if self._unread else self._last
        out = (capi.Result * max(n, 1))()
        check(lib.s2_batch_results(self._h, out, n), "results")
        return [(r.score, np.array(r.stats[:]), np.array(r.sums[:]), r.n_scales, r.status, r.dssim,
                 np.array(r.dssim_scale[:])) for r in out[:n]]

    def compute_batch(self, pairs, stream=None):
        self.submit(pairs, stream)
        return self.results()

    # ---- cached reference: ssim2-gpu Ssim2Batch (pipeline_batch.rs:206-330) ----
    def set_reference(self, ref, fmt="srgb8", ref_uv=None, stream=None, **kw):
        """Cache the reference (a device tensor of any supported format)."""
        d = PairDesc(ref, ref, fmt, ref_uv, ref_uv, **kw).to_c()
        d.dis = d.dis_uv = None
        self._ref_keep = (ref, ref_uv)
        check(lib.s2_batch_set_reference(self._h, ctypes.byref(d), _stream_ptr(stream)), "set_reference")

    def clear_reference(self):
        check(lib.s2_batch_clear_reference(self._h), "clear_reference")

    def has_cached_reference(self):
        return bool(lib.s2_batch_has_reference(self._h))

    def submit_with_reference(self, dis, fmt="srgb8", dis_uv=None, stream=None, **kw):
        """Enqueue distorted images (device tensors, one size) against the
        cached reference; `dis_uv` gives their CbCr planes for 4:2:0 input."""
        arr = (capi.PairDescC * max(len(dis), 1))()
        for i, t in enumerate(dis):
            arr[i] = PairDesc(t, t, fmt, dis_uv[i] if dis_uv else None, dis_uv[i] if dis_uv else None, **kw).to_c()
            arr[i].ref = arr[i].ref_uv = None
        k = self._take_slot(False)
        check(lib.s2_batch_submit_with_reference(self._h, arr, len(dis), _stream_ptr(stream)), "compute_batch")
        self._last = (k, len(dis), (dis, dis_uv))
        self._unread.append(self._last)

    def compute_batch_with_reference(self, dis, fmt="srgb8", dis_uv=None, stream=None, **kw):
        self.submit_with_reference(dis, fmt, dis_uv, stream, **kw)
        return self.results()

    def mem_usage(self):
        n = ctypes.c_size_t()
        check(lib.s2_batch_mem_usage(self._h, ctypes.byref(n)), "mem_usage")
        return n.value


class Dssim:
    """DSSIM of one size: the drop-in for dssim-cuda's `Dssim`
    (crates/dssim-cuda/src/lib.rs:170-467).  Images are sRGB8 (H, W, 3):
    torch CUDA tensors, or host arrays for the `*_from_cpu` calls."""

    def __init__(self, width, height, *, device=0):
        self.width, self.height = int(width), int(height)
        h = ctypes.c_void_p()
        check(lib.s2_dssim_create(device, self.width, self.height, ctypes.byref(h)), "Dssim::new")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.s2_dssim_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def compute_sync(self, ref_srgb, dis_srgb, stream=None):
        """Dssim::compute_sync (lib.rs:225-232)."""
        rp, rpitch = _dev(ref_srgb, 1)
        dp, dpitch = _dev(dis_srgb, 1)
        v = ctypes.c_double()
        check(lib.s2_dssim_compute_srgb8(self._h, rp, rpitch, dp, dpitch, 0, _stream_ptr(stream), ctypes.byref(v)),
              "Dssim::compute_sync")
        return v.value

    def compute_sync_dis_only(self, dis_srgb, stream=None):
        """Dssim::compute_sync_dis_only (lib.rs:245-251): against the reference
        of the last compute_sync."""
        dp, dpitch = _dev(dis_srgb, 1)
        v = ctypes.c_double()
        check(lib.s2_dssim_compute_dis_only_srgb8(self._h, dp, dpitch, 0, _stream_ptr(stream), ctypes.byref(v)),
              "Dssim::compute_sync_dis_only")
        return v.value

    def compute_from_cpu_sync(self, ref_bytes, dis_bytes, stream=None):
        """Host sRGB8 (H, W, 3) pair (uploaded by the library)."""
        rp, rpitch, _ = _host(ref_bytes)
        dp, dpitch, _ = _host(dis_bytes)
        v = ctypes.c_double()
        check(lib.s2_dssim_compute_srgb8(self._h, rp, rpitch, dp, dpitch, 1, _stream_ptr(stream), ctypes.byref(v)),
              "Dssim::compute_from_cpu_sync")
        return v.value

    def mem_usage(self):
        """Dssim::mem_usage (lib.rs:438-451)."""
        n = ctypes.c_size_t()
        check(lib.s2_dssim_mem_usage(self._h, ctypes.byref(n)), "mem_usage")
        return n.value


class Zensim:
    """zensim's 228-feature extraction of one size: the drop-in for
    zensim-cuda's `Zensim` (crates/zensim-cuda/src/lib.rs:168-819).  Images
    are packed sRGB8 (H, W, 3): torch CUDA tensors, or host arrays for the
    `*_from_cpu` calls.  The score needs the trained weight table of the zensim
    crate, which the reference tree does not hold: features only."""

    FEATURES = 228

    def __init__(self, width, height, *, device=0):
        self.width, self.height = int(width), int(height)
        h = ctypes.c_void_p()
        check(lib.s2_zensim_create(device, self.width, self.height, ctypes.byref(h)), "Zensim::new")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.s2_zensim_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def _img(self, img, on_host):
        if on_host:
            p, pitch, keep = _host(img)
            return p, pitch, keep
        p, pitch = _dev(img, 1)
        return p, pitch, None

    def set_reference(self, ref_srgb, on_host=False, stream=None):
        """Zensim::set_reference (lib.rs:340-376)."""
        p, pitch, _ = self._img(ref_srgb, on_host)
        check(lib.s2_zensim_set_reference_srgb8(self._h, p, pitch, 1 if on_host else 0, _stream_ptr(stream)),
              "Zensim::set_reference")

    def compute_with_reference(self, dis_srgb, on_host=False, stream=None):
        """Zensim::compute_with_reference (lib.rs:388-395): 228 features."""
        p, pitch, _ = self._img(dis_srgb, on_host)
        feat = np.zeros(self.FEATURES)
        ns = ctypes.c_int32()
        check(lib.s2_zensim_compute_with_reference_srgb8(self._h, p, pitch, 1 if on_host else 0, _stream_ptr(stream),
                                                         feat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                         ctypes.byref(ns)), "Zensim::compute_with_reference")
        self.n_scales = ns.value
        return feat

    def compute_features(self, ref_srgb, dis_srgb, on_host=False, stream=None):
        """Zensim::compute_features (lib.rs:322-329)."""
        self.set_reference(ref_srgb, on_host, stream)
        return self.compute_with_reference(dis_srgb, on_host, stream)

    def has_reference(self):
        return bool(lib.s2_zensim_has_reference(self._h))

    def clear_reference(self):
        check(lib.s2_zensim_clear_reference(self._h), "Zensim::clear_reference")

    def raw(self):
        """Zensim::debug_compute_raw's sums of the last compute: acc (4, 3, 17)
        and the maxima (4, 3, 3) as float32."""
        acc = np.zeros((4, 3, 17))
        peaks = np.zeros((4, 3, 3), np.uint32)
        check(lib.s2_zensim_raw(self._h, acc.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                peaks.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))), "raw")
        return acc, peaks.view(np.float32)

    def mem_usage(self):
        n = ctypes.c_size_t()
        check(lib.s2_zensim_mem_usage(self._h, ctypes.byref(n)), "mem_usage")
        return n.value
