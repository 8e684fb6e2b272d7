// Runner for the reference's own GPU path: build_rtree
// (src/rtree_bulkload_thrust.cuh:62) and bfs_frontier
// (src/rtree_bfs_frontier.cuh:292), compiled from the reference sources where
// they lie into oracle/_ref/ref_frontier by oracle/Makefile.
// TEST INFRASTRUCTURE ONLY: it writes the golden node arrays and hit pairs
// the oracle is pinned against, and times the reference's GPU path as a
// reported baseline.
//
//   ref_frontier build <boxes.crtb> - <fanout> <outdir> <reps>
//   ref_frontier query <boxes.crtb> <queries.crtb> <fanout> <outdir> <reps>
//
// Outputs in <outdir>: tree.bin (int64 R_sz, int64 fanout, then R_sz float32
// xmin/ymin/xmax/ymax and int32 pos/len), sorted_ids.bin (int32 id per sorted
// slot), pairs.bin (int64 count, then int32 fid[] and tid[]) for `query`.
// One line "REFJSON {...}" on stdout carries the timings.
#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>
#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/iterator/constant_iterator.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/discard_iterator.h>
#include <thrust/iterator/transform_iterator.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/merge.h>
#include <thrust/reduce.h>
#include <thrust/remove.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/tuple.h>
#include <time.h>
#include <iostream>
#include <string>
#include <vector>

#include "rtree.h"
#include "rtree_bfs_frontier.cuh"
#include "rtree_bulkload_thrust.cuh"
#include "utility.cuh"
#include "utility.h"

#include "crtb_io.h"

#define REF_QUERY_FN bfs_frontier
#define REF_IMPL_NAME "frontier"
#include "ref_runner_main.inc"
