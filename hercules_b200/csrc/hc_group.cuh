// hc_group.cuh -- one launch of a kernel over the blocks of many channels.
//
// Every kernel of the FD step is a __device__ body that takes its block index
// and grid as arguments (named blockIdx and gridDim, so the body reads them as
// it would the built-ins) plus a __global__ wrapper that passes the built-ins.
// k_group runs the same body for a list of channels in one launch: the blocks
// of the 1-D launch are the concatenated grids of the members, and each block
// finds its member (binary search over the prefix sums of the members' block
// counts), its block index in that member's grid, and the member's arguments in
// a device table. Every member's block then does exactly what it does in the
// member's own launch, so the results are the same bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <string.h>
#include <vector>

template <typename A> struct GroupTab {
    int n;                 // members
    const int* start;      // n+1 prefix sums of the members' block counts
    const dim3* grid;      // the members' own grids
    const A* args;         // the members' arguments
};

template <typename A, void (*BODY)(const A&, const uint3, const dim3), int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_group(GroupTab<A> t)
{
    const int b = blockIdx.x;
    int lo = 0, hi = t.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(t.start + mid) <= b) lo = mid; else hi = mid - 1;
    }
    const dim3 gd = t.grid[lo];
    const int lb = b - __ldg(t.start + lo);
    uint3 bi;
    bi.x = lb % gd.x;
    bi.y = (lb / gd.x) % gd.y;
    bi.z = lb / (gd.x * gd.y);
    BODY(t.args[lo], bi, gd);
}

struct GroupLaunch;

// One recorded launch of one channel: the grouped kernel that can run its body
// (which identifies the kernel variant), how to build a group of such launches,
// and the launch's own arguments and shape.
struct GroupRec {
    const void* key;
    int (*build)(const GroupRec* const* recs, int n, GroupLaunch* out);
    std::vector<unsigned char> args;
    dim3 grid, block;
    size_t smem;
};

// A built group: its device table (one allocation) and how to launch it.
struct GroupLaunch {
    void (*run)(const GroupLaunch& g, cudaStream_t st);
    void* dbuf;
    int n;
    unsigned nblk;
    dim3 block;
    size_t smem;
    const void* args;
    const int* start;
    const dim3* grid;
};

template <typename A, void (*BODY)(const A&, const uint3, const dim3), int NT, int MINB>
static void group_run(const GroupLaunch& gl, cudaStream_t st)
{
    GroupTab<A> t;
    t.n = gl.n; t.start = gl.start; t.grid = gl.grid; t.args = (const A*)gl.args;
    k_group<A, BODY, NT, MINB><<<gl.nblk, gl.block, gl.smem, st>>>(t);
}

static inline size_t group_align(size_t x) { return (x + 255) & ~(size_t)255; }

// Build the device table of a group of recorded launches of the same body.
// Returns 0, or -1 if the members' block shapes differ or the table cannot be
// allocated (the caller then runs the members apart).
template <typename A, void (*BODY)(const A&, const uint3, const dim3), int NT, int MINB>
static int group_build(const GroupRec* const* recs, int n, GroupLaunch* out)
{
    std::vector<int> start(n + 1);
    std::vector<dim3> grid(n);
    std::vector<unsigned char> args((size_t)n * sizeof(A));
    long long tot = 0;
    size_t smem = 0;
    const dim3 blk = recs[0]->block;
    for (int m = 0; m < n; ++m) {
        const GroupRec& r = *recs[m];
        if (r.block.x != blk.x || r.block.y != blk.y || r.block.z != blk.z || r.args.size() != sizeof(A)) return -1;
        start[m] = (int)tot;
        grid[m] = r.grid;
        memcpy(args.data() + (size_t)m * sizeof(A), r.args.data(), sizeof(A));
        tot += (long long)r.grid.x * r.grid.y * r.grid.z;
        if (r.smem > smem) smem = r.smem;
    }
    if (tot > 0x7fffffffLL) return -1;
    start[n] = (int)tot;
    const size_t oa = 0, os = group_align((size_t)n * sizeof(A)), og = os + group_align((size_t)(n + 1) * sizeof(int));
    const size_t total = og + (size_t)n * sizeof(dim3);
    unsigned char* d = nullptr;
    if (cudaMalloc(&d, total) != cudaSuccess) return -1;
    if (cudaMemcpy(d + oa, args.data(), args.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d + os, start.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d + og, grid.data(), n * sizeof(dim3), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return -1;
    }
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_group<A, BODY, NT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaFree(d);
        return -1;
    }
    out->run = &group_run<A, BODY, NT, MINB>;
    out->dbuf = d;
    out->n = n;
    out->nblk = (unsigned)tot;
    out->block = blk;
    out->smem = smem;
    out->args = d + oa;
    out->start = (const int*)(d + os);
    out->grid = (const dim3*)(d + og);
    return 0;
}
