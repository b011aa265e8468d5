"""B200-native (sm_100a) implementation of gkmsvm-lite's pairwise gapped-k-mer
kernel path: GkmSVM scoring, score_variants, ISM, GkmExplain, the training
Gram matrix and the SMO solver's kernel columns, with the reference's signatures, computed by hand-written CUDA
kernels behind the C ABI of include/gkm_b200.h."""

from .deltasvm import DeltaSVMWeights, deltasvm_weights
from .explain import gkmexplain, mutation_impact
from .gram import compute_gram
from .importers import load_classic_model, load_lsgkm_model, load_r_gkmsvm_model, parse_lsgkm_header, read_fasta
from .inputs import as_batch, encode_codes, to_codes
from .ism import ism
from .kernels import (KERNEL_ALIASES, KERNEL_BUILDERS, CenterWeightedGkmKernel, CenterWeightedRbfGkmKernel,
                      DirectGkmKernel, EstTruncGkmKernel, GkmKernel, RbfGkmKernel, RbfKernel,
                      resolve_kernel_type)
from .model import GkmSVM
from .serialization import (load_deltasvm_npz, load_model, load_npz, save_deltasvm_npz, save_lsgkm,
                            save_npz)
from .solver import KernelColumnCache, smo_solve, smo_svr_solve

__all__ = [
    "GkmSVM", "ism", "gkmexplain", "mutation_impact", "compute_gram", "load_lsgkm_model", "load_model",
    "KERNEL_ALIASES", "KERNEL_BUILDERS", "resolve_kernel_type", "GkmKernel", "DirectGkmKernel",
    "EstTruncGkmKernel", "CenterWeightedGkmKernel", "RbfKernel", "RbfGkmKernel",
    "CenterWeightedRbfGkmKernel", "as_batch", "encode_codes", "to_codes", "KernelColumnCache", "smo_solve",
    "smo_svr_solve", "DeltaSVMWeights", "deltasvm_weights", "parse_lsgkm_header", "load_npz", "save_npz",
    "save_lsgkm", "load_deltasvm_npz", "save_deltasvm_npz", "load_classic_model", "load_r_gkmsvm_model", "read_fasta",
]
