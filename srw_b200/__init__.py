"""srw_b200: SRW's Fourier-optics wavefront propagation (srwlPropagElecField over drift / thin
lens / aperture chains) as hand-written sm_100a kernels behind the reference's C API.

    from srw_b200 import srwlpy as srwl        # drop-in for srwlpy.PropagElecField
    from srw_b200.srwlib import SRWLWfr, SRWLOptD, SRWLOptA, SRWLOptL, SRWLOptC
    from srw_b200.plan import Plan             # device-resident planning / batched execution
"""
from . import capi  # noqa: F401

__all__ = ['capi', 'srwlib', 'srwlpy']
