// batch.h -- the batched-evaluation object (instances, offsets, work queues, schedules),
// shared by the batched kernels (batch.cu) and the per-instance solves (solve.cu).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <utility>
#include <vector>

#include "handle.h"

namespace bosss {
struct BatchInst;
struct WorkItem;
}  // namespace bosss

struct bosss_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    int phys = 0, D = 0, n = 0;
    std::vector<bosss_handle*> h;                 // per-instance descriptors (tables, grid, physics)
    std::vector<long long> dom_off, cod_off;      // n+1 prefix offsets
    bosss::BatchInst* d_inst = nullptr;
    bosss::WorkItem* d_items[3] = {nullptr, nullptr, nullptr};
    int nitems[3] = {0, 0, 0};
    int* d_counter = nullptr;                     // two queue counters (two kernels per graph)
    int grid[3] = {0, 0, 0};
    std::map<std::pair<int, int>, int> tiles;     // (K, Q) -> tiles per work item (autotuned)
    bool slab[3] = {false, false, false};         // tile kernel per mode: slab or generic
    bool lpt = true;                              // longest-processing-time-first order
    // per-class schedule (one launch per (K, Q) class and mode) instead of the persistent queue
    struct ClassRun {
        int K, Q;
        bool slab;
        int first, count;   // range of this class's tiles in d_class_items[mode]
    };
    bool classes = false;
    std::vector<ClassRun> runs[3];
    bosss::WorkItem* d_class_items[3] = {nullptr, nullptr, nullptr};
    cudaGraphExec_t graph = nullptr;
};
