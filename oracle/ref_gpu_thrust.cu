// Runner for the reference's own GPU path with the Thrust BFS: build_rtree
// (src/rtree_bulkload_thrust.cuh:62) and bfs_thrust
// (src/rtree_bfs_thrust.cuh:59), compiled from the reference sources where
// they lie, against the small RMM stand-in under oracle/rmm_shim, into
// oracle/_ref/ref_thrust by oracle/Makefile.  Same command line and outputs
// as oracle/ref_gpu_frontier.cu.  TEST INFRASTRUCTURE ONLY.
#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>
#include <iostream>
#include <iterator>
#include <string>
#include <vector>

#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/equal.h>
#include <thrust/execution_policy.h>
#include <thrust/host_vector.h>
#include <thrust/iterator/constant_iterator.h>
#include <thrust/reduce.h>
#include <thrust/sequence.h>
#include <thrust/scatter.h>
#include <thrust/scan.h>
#include <thrust/uninitialized_fill.h>

#include "rtree.h"
#include "rtree_bfs_thrust.cuh"
#include "rtree_bulkload_thrust.cuh"
#include "utility.cuh"
#include "utility.h"

#include "crtb_io.h"

#define REF_QUERY_FN bfs_thrust
#define REF_IMPL_NAME "thrust"
#include "ref_runner_main.inc"
