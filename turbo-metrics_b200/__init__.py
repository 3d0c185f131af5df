"""turbo-metrics B200: SSIMULACRA2 (and DSSIM from the same pyramid) on
sm_100a behind a C ABI.

Python host mirror of the `ssimulacra2-cuda` crate's `Ssimulacra2` type
(crates/ssimulacra2-cuda/src/lib.rs:27-602) and of `ssim2-gpu`'s batch API
(crates/ssim2-gpu/src/pipeline_batch.rs:120-382), bound with ctypes to
libssim2b200.so (include/ssim2b200.h).  Method names, argument meaning and
error cases follow the reference; errors are exceptions instead of panics.

Device buffers are passed as torch CUDA tensors (or as `(pointer, pitch)`
tuples); torch is only the allocator and stream provider here.  There is no
CPU fallback: importing this package without the built library raises.
"""
from .capi import (  # noqa: F401
    S2Error,
    Busy,
    Timeout,
    InvalidArgument,
    InvalidImageSize,
    DimensionMismatch,
    NoCachedReference,
    OutOfMemory,
    lib,
    library_path,
    num_scales,
    version,
)
from .ssimulacra2 import Ssimulacra2, Ssim2Batch, PairDesc, Dssim, Zensim  # noqa: F401
from .server import Ssim2Server  # noqa: F401
from .frames import FramePairScorer, Stats, select_frames  # noqa: F401
from .router import RoutingPolicy, FrontEnd, Job, ServerEngine, worker_loop  # noqa: F401
