"""rotormap -- B200-native host API of RotorMap's read-mapping hot path.

The names mirror the reference's Julia entry points (RotorMap/encode,
index, search, tools/map.jl); every device operation is a call into
librotormap_b200.so (C ABI: include/r2m.h).  There is no CPU fallback.
"""
from ._lib import R2MError, lib, require_device
from .encoder import (RopeEncoder, dim, encode_frag_real_batch, encode_frag_real_batch_alloc,
                      f16_to_f8, f32_to_f8, revcomp_frag_words)
from .engine import (CompactEngine, Mapper, PlainEngine, TopKBatch, TopKEngine, batch_gemm_topk, padmul, resident_fits,
                     rope_topk_stream, rope_topk_stream_compact, topk_flow, upload_fp16_as_f8)
from .fasta import (DeviceFastaFragments, FastaFragments, HeaderList, fasta_chunks_device, fasta_reads,
                    fasta_reads_device)
from .index import (FP8_FORMAT, ROW_FORMAT, SCALED_FORMAT, Index, RefPack, attach_genome, build_index,
                    build_index_packed, index_database, index_to_f8, load_index, pack_records,
                    pack_reference, save_index, window_positions)
from . import jlbin
from .batching import Autotuner, RaggedBatcher, bucket_rows
from .precision import DeviceMeta, check_fp64, map_precise, rescore_fp32
from .mapping import julia_repr_f32, map_and_count, parse_read_head, run_map, score_provenance

__all__ = [n for n in dir() if not n.startswith("_")]
