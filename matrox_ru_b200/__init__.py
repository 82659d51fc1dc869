"""B200-native evaluator of MatRox's hot path: Y = K~ W for HSS / H2-b compressed kernel
matrices given in MatRox's compressed data storage (CDS).

Modules:
  structure  host-side CDS producer (tree, interaction lists, ID compression) in the
             reference's array layout
  hgemm      the reference-signature drop-ins, device plans and the evaluator
  autograd   torch.autograd.Function with the transposed traversal as backward
  build      nvcc build of libmatrox_b200.so (sm_100a)
"""
from .structure import CDS, KernelSpec, build_cds, gaussian_mixture  # noqa: F401

__all__ = ["CDS", "KernelSpec", "build_cds", "gaussian_mixture"]
