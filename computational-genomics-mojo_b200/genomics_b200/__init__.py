"""genomics_b200: B200 (sm_100a) batched pairwise alignment.

Host-side mirror of the reference's alignment interface
(genomics/core/{dna,sequence}.mojo, genomics/cpu/align_cpu.mojo,
genomics/gpu/{device,align_gpu}.mojo) over the C ABI of libgenomics_b200.so.
"""
from .core import (BASES_PER_WORD, Base, NMask, SequenceBatch, SequenceView, ascii_to_2bit,
                   base_to_ascii, get_base_from_word, get_view, pack_ascii)
from .align import (AlignConfig, AlignResult, WFAConfig, default_config, default_wfa_config,
                    needleman_wunsch_banded, smith_waterman_banded, sw_banded_batch, wfa_affine,
                    wfa_affine_batch, wfa_affine_cigar_cpu, wfa_affine_cpu)
from .device import DeviceBatch, GenomicsDevice, launch_banded_sw, launch_wfa_affine
from ._lib import GenomicsError

__version__ = "0.1.0"
