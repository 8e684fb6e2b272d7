"""crtree-b200: a B200-native 2-D bounding-box R-tree (Z-order bulk load and
batched window query) behind the C ABI declared in include/crtree.h.

Python mirror of the reference interface (trxcllnt/curtree src/rtree.h,
src/rtree_bulkload_thrust.cuh, src/rtree_bfs_frontier.cuh,
src/rtree_bfs_thrust.cuh): BBox, RTree, IDPair, build_rtree, bfs_frontier,
bfs_thrust, read_mbr_csv; plus the extended query API (query_into, query,
query_stream, Plan).
"""
from . import datasets
from ._lib import CRT_QUERY_PERSISTENT, CRT_QUERY_PLAIN, CrtError
from .rtree import (BBox, IDPair, PairDigest, Plan, RTree, bfs_frontier, bfs_thrust, build_into, build_rtree,
                    canonicalize,
                    kernel_launches, new_result_block, query, query_capacity, query_into,
                    query_stats, query_stream, read_mbr_bin, read_mbr_csv, read_result, tree_size)

__all__ = ["datasets", "BBox", "RTree", "IDPair", "PairDigest", "Plan", "build_rtree", "build_into", "canonicalize",
           "bfs_frontier", "bfs_thrust", "query", "query_into", "query_stats", "query_stream", "query_capacity", "tree_size",
           "new_result_block", "read_result", "read_mbr_csv", "read_mbr_bin", "kernel_launches", "CrtError",
           "CRT_QUERY_PERSISTENT", "CRT_QUERY_PLAIN"]
