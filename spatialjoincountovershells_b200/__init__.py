"""B200-native spatial join count over shells (SJCS) hot path.

Python access to the two native libraries of this package:

* ``libsjcs.so`` -- the GPU path (index build + periodic multi-shell count) behind
  the C ABI of ``include/sjcs.h``.  There is no CPU fallback: every call that
  computes needs a CUDA device and raises :class:`SjcsError` otherwise, and
  importing the GPU API raises if the library was not built.
* ``libsjcs_host.so`` -- the reference's file formats and the seeded data
  generators (``include/sjcs_host.h``); CPU only.

The call sequence mirrors the reference driver's (src/astr_rcount/main.c):
build an index per particle file (constructArraySTR + makeTree*), count every
halo's shells against it (multiRangeCountWithPriodicBoundArraySTR per halo in
threadJoin), accumulate across files, destroy the index.
"""
from __future__ import annotations

from ._native import (  # noqa: F401
    HALO_DTYPE,
    INDEX_GRID,
    INDEX_LEARNED,
    INDEX_MORTON,
    INDEX_VERIFY,
    QUERY_NONPERIODIC,
    QUERY_PERIODIC,
    SCHED_AUTO,
    SCHED_QUEUE,
    SCHED_STATIC,
    Context,
    Index,
    Query,
    Server,
    SjcsError,
    gen_clustered_halos,
    gen_clustered_particles,
    gen_face_halos,
    gen_uniform_halo_file,
    gen_uniform_halos,
    gen_uniform_particles,
    host_lib,
    host_lib_path,
    lib,
    lib_path,
    multi_range_count_with_periodic_bound,
    radius_table,
    read_halos,
    read_particles,
    write_halo_file,
    write_particle_file,
    write_result,
)

__all__ = [
    "Context", "Index", "Query", "SjcsError", "radius_table", "read_halos", "read_particles",
    "write_result", "multi_range_count_with_periodic_bound",
]
