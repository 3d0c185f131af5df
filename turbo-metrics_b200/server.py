"""`Ssim2Server`: continuous-batching SSIMULACRA2 server over the C ABI.

Jobs are one host sRGB8 reference plus k host sRGB8 candidates of the same
size (an encoder's quality search).  The native worker admits jobs in arrival
order under the HBM budget, uploads them on a copy stream and scores the
pending work of all admitted jobs in each round; a job's reference pyramid is
built once.  See the s2_server_* section of include/ssim2b200.h.
"""
import ctypes

import numpy as np

from . import capi
from .capi import lib, check


class Ssim2Server:
    def __init__(self, device=0, max_batch_pairs=256, max_batch_pixels=32 << 20, hbm_budget=40 << 30,
                 max_queued_jobs=None):
        """max_queued_jobs: unfinished jobs beyond which submit raises Busy
        (None: the library default, 128)."""
        cfg = capi.ServerConfig()
        lib.s2_server_config_default(ctypes.byref(cfg))
        cfg.device, cfg.max_batch_pairs, cfg.max_batch_pixels = device, max_batch_pairs, max_batch_pixels
        cfg.hbm_budget = hbm_budget
        if max_queued_jobs is not None:
            cfg.max_queued_jobs = max_queued_jobs
        h = ctypes.c_void_p()
        check(lib.s2_server_create(ctypes.byref(cfg), ctypes.byref(h)), "Ssim2Server")
        self._h = h
        self._keep = {}

    @staticmethod
    def _rows(a):
        """An (H, W, 3) uint8 image whose rows are packed pixels, as is (a crop
        of a larger image keeps its row pitch), else a packed copy."""
        if a.dtype == np.uint8 and a.ndim == 3 and a.shape[2] == 3 and a.strides[2] == 1 and a.strides[1] == 3 \
                and a.strides[0] >= 3 * a.shape[1]:
            return a
        return np.ascontiguousarray(a, np.uint8)

    def submit(self, ref, candidates):
        """ref, candidates: (H, W, 3) uint8 host arrays (crops of larger
        images are passed with their row pitch, not copied).  Returns a job
        id; raises Busy when the server holds max_queued_jobs unfinished
        jobs."""
        ref = self._rows(ref)
        cands = [self._rows(c) for c in candidates]
        for c in cands:
            if c.shape != ref.shape:
                raise capi.DimensionMismatch(capi.S2_ERR_DIM_MISMATCH, "submit")
        pitch = cands[0].strides[0] if cands else ref.strides[0]
        if any(c.strides[0] != pitch for c in cands):
            cands = [np.ascontiguousarray(c) for c in cands]
            pitch = cands[0].strides[0]
        arr = (ctypes.c_void_p * max(len(cands), 1))(*[c.ctypes.data for c in cands])
        jd = capi.JobDesc()
        jd.height, jd.width = ref.shape[0], ref.shape[1]
        jd.format = capi.FMT["srgb8"]
        jd.ref, jd.ref_pitch = ref.ctypes.data, ref.strides[0]
        jd.n_candidates = len(cands)
        jd.candidates = ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p))
        jd.cand_pitch = pitch
        jid = ctypes.c_uint64()
        check(lib.s2_server_submit(self._h, ctypes.byref(jd), ctypes.byref(jid)), "submit")
        self._keep[jid.value] = (ref, cands, arr)  # host images must outlive the job
        return jid.value

    def wait(self, job_id, timeout_ms=60000):
        """(scores, statuses, latency_ms); raises on timeout / cancellation."""
        n = len(self._keep[job_id][1])
        sc = np.zeros(max(n, 1))
        st = np.zeros(max(n, 1), np.int32)
        lat = ctypes.c_double()
        rc = lib.s2_server_wait(self._h, job_id, timeout_ms, sc.ctypes.data_as(capi.D),
                                st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(lat))
        if rc != capi.S2_ERR_TIMEOUT:
            self._keep.pop(job_id, None)
        check(rc, "wait")
        return sc[:n], st[:n], lat.value

    def cancel(self, job_id):
        check(lib.s2_server_cancel(self._h, job_id), "cancel")

    def stats(self):
        r = capi.ServerReport()
        check(lib.s2_server_stats(self._h, ctypes.byref(r)), "stats")
        return {f: getattr(r, f) for f, _ in capi.ServerReport._fields_}

    def reset_stats(self):
        check(lib.s2_server_reset_stats(self._h), "reset_stats")

    def close(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.s2_server_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()
