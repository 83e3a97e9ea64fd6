// hc_group.cuh -- one launch of a kernel over the blocks of many channels.
//
// Every kernel of the FD step is a __device__ body that takes its block index
// and grid as arguments (named blockIdx and gridDim, so the body reads them as
// it would the built-ins) plus a __global__ wrapper that passes the built-ins.
// k_group runs the same body for a list of channels in one launch: the blocks
// of the 1-D launch are the concatenated grids of the members, and each block
// finds its member (binary search over the prefix sums of the members' block
// counts), its block index in that member's grid, and the member's arguments in
// the launch's parameter block. Every member's block then does exactly what it
// does in the member's own launch. The table is a __grid_constant__ parameter, so
// the body reads its arguments from the constant bank as in its own kernel (read
// from global memory they may alias the kernel's stores, which changed how the
// compiler contracted FP32 products). The grouped kernel is still a separate
// compilation of the body: FP64 results have matched the member's own launches
// bit for bit, FP32 ones agree to a few units in the last place where the
// compiler fused a multiply and an add differently.
#pragma once
#include <cuda_runtime.h>
#include <string.h>
#include <vector>

// Members a grouped launch carries in its parameter block (kernel parameters may
// take up to 32 KB on this architecture).
template <typename A> struct GroupCap {
    static constexpr int v = (32000 - 16) / (int)(sizeof(A) + sizeof(int) + sizeof(dim3)) < 64
                                 ? (32000 - 16) / (int)(sizeof(A) + sizeof(int) + sizeof(dim3)) : 64;
};

// The table of a grouped launch, passed as the kernel's parameter block: the
// members' arguments are read from the constant bank, as in their own kernels.
// Two capacities: up to 8 members (a few KB of parameters a launch) and up to
// GroupCap<A> members.
#define HC_GROUP_SMALL 8
template <typename A> struct GroupSmall {
    static constexpr int v = HC_GROUP_SMALL < GroupCap<A>::v ? HC_GROUP_SMALL : GroupCap<A>::v;
};
// Raise a kernel's dynamic shared-memory limit to what the device allows next to
// the kernel's own static shared memory (the same limit from every call site).
static inline cudaError_t group_raise_smem(const void* kernel)
{
    int dev = 0, optin = 0;
    cudaFuncAttributes fa;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    return e;
}
template <typename A, int CAP> struct GroupTab {
    int n;                 // members
    int start[CAP + 1];    // prefix sums of the members' block counts
    dim3 grid[CAP];        // the members' own grids
    A args[CAP];           // the members' arguments
};

template <typename A, void (*BODY)(const A&, const uint3, const dim3), int NT, int MINB, int CAP>
__global__ void __launch_bounds__(NT, MINB) k_group(const __grid_constant__ GroupTab<A, CAP> t)
{
    const int b = blockIdx.x;
    int lo = 0, hi = t.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.start[mid] <= b) lo = mid; else hi = mid - 1;
    }
    const dim3 gd = t.grid[lo];
    const int lb = b - t.start[lo];
    uint3 bi;
    bi.x = lb % gd.x;
    bi.y = (lb / gd.x) % gd.y;
    bi.z = lb / (gd.x * gd.y);
    BODY(t.args[lo], bi, gd);
}

struct GroupLaunch;

// One recorded launch of one channel: the grouped kernel that can run its body
// (which identifies the kernel variant), the most members one grouped launch
// takes, how to build a group of such launches, and the launch's own arguments
// and shape.
struct GroupRec {
    const void* key;
    int cap;
    int (*build)(const GroupRec* const* recs, int n, GroupLaunch* out);
    std::vector<unsigned char> args;
    dim3 grid, block;
    size_t smem;
};

// A built group: its parameter block and how to launch it.
struct GroupLaunch {
    void (*run)(const GroupLaunch& g, cudaStream_t st);
    int pos;               // position in the members' launch sequences
    unsigned nblk;
    dim3 block;
    size_t smem;
    std::vector<unsigned char> params;
};

template <typename A, void (*BODY)(const A&, const uint3, const dim3), int NT, int MINB, int CAP>
static void group_run(const GroupLaunch& gl, cudaStream_t st)
{
    k_group<A, BODY, NT, MINB, CAP><<<gl.nblk, gl.block, gl.smem, st>>>(
        *reinterpret_cast<const GroupTab<A, CAP>*>(gl.params.data()));
}

// Build a grouped launch of at most GroupCap<A> recorded launches of the same
// body. Returns 0, or -1 if the members' block shapes differ (the caller then
// runs the members apart).
template <typename A, void (*BODY)(const A&, const uint3, const dim3), int NT, int MINB, int CAP>
static int group_build_cap(const GroupRec* const* recs, int n, GroupLaunch* out)
{
    if (n < 1 || n > CAP) return -1;
    out->params.assign(sizeof(GroupTab<A, CAP>), 0);
    GroupTab<A, CAP>* t = reinterpret_cast<GroupTab<A, CAP>*>(out->params.data());
    long long tot = 0;
    size_t smem = 0;
    const dim3 blk = recs[0]->block;
    t->n = n;
    for (int m = 0; m < n; ++m) {
        const GroupRec& r = *recs[m];
        if (r.block.x != blk.x || r.block.y != blk.y || r.block.z != blk.z || r.args.size() != sizeof(A)) return -1;
        t->start[m] = (int)tot;
        t->grid[m] = r.grid;
        memcpy(&t->args[m], r.args.data(), sizeof(A));
        tot += (long long)r.grid.x * r.grid.y * r.grid.z;
        if (r.smem > smem) smem = r.smem;
    }
    if (tot > 0x7fffffffLL) return -1;
    t->start[n] = (int)tot;
    // the same limit a channel's own launches set (a lower one would refuse them)
    if (smem > 48 * 1024 && group_raise_smem((const void*)k_group<A, BODY, NT, MINB, CAP>) != cudaSuccess)
        return -1;
    out->run = &group_run<A, BODY, NT, MINB, CAP>;
    out->nblk = (unsigned)tot;
    out->block = blk;
    out->smem = smem;
    return 0;
}

template <typename A, void (*BODY)(const A&, const uint3, const dim3), int NT, int MINB>
static int group_build(const GroupRec* const* recs, int n, GroupLaunch* out)
{
    if (n <= GroupSmall<A>::v) return group_build_cap<A, BODY, NT, MINB, GroupSmall<A>::v>(recs, n, out);
    return group_build_cap<A, BODY, NT, MINB, GroupCap<A>::v>(recs, n, out);
}
