/*
 * gcomcot_fused_step_noalloc: one fused linear-spherical time step over a
 * caller-supplied list of grids, for callers that cannot allocate device
 * memory.
 *
 * Who needs it: codes that own every byte of device memory themselves and
 * forbid library allocations (a Fortran model that sizes its arrays once at
 * start-up, an operational warning pipeline that reserves a fixed memory budget
 * before the first alert arrives), and time-critical loops in which an
 * allocation is not acceptable because it may synchronise the device or fail
 * under memory pressure.  The batched engine takes its work list from the
 * stream-ordered allocator; this entry point keeps the same work list in a
 * fixed array compiled into the library instead.
 *
 * The scratch is one file-scope __device__ array of GC_NOALLOC_SCRATCH_BYTES
 * (about 200 KB).  Every GPU that loads this library holds it until the process
 * exits.  It holds at most GC_NOALLOC_MAX_GRIDS grid descriptors and
 * GC_NOALLOC_MAX_TILES tiles; larger requests are rejected.
 *
 * Nothing is copied from host memory: the grid descriptors travel to the GPU
 * inside the launch parameters of a small kernel (k_noalloc_fill, one
 * __grid_constant__ block of about 13 KB), which writes them and the tile work
 * list into the scratch; the fused step then reads them from there, in stream
 * order.  A call therefore returns as soon as its two kernels are queued.
 * Every call overwrites all the scratch entries it uses before its step reads
 * them, so nothing in the scratch has to start at zero -- and two calls whose
 * work overlaps on the GPU (different streams, or different host threads) race
 * on it: issue them one after the other on one stream.
 *
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress with that device current) and sets the fused kernel's
 * shared-memory limit on that device; make that first call before any stream
 * capture.
 *
 * Bounded waits: a pipeline wait of the fused kernel that gives up sets the
 * library's error flag.  Each call clears the flag, in stream order, before
 * its step; after synchronising its stream the caller reads (and clears) it
 * with gcomcot_sync(), which then returns GC_ETIMEOUT.
 */
#include <mutex>
#include <string.h>

#include "fused.h"
#include "gcomcot.h"

#define GC_NOALLOC_MAX_GRIDS 64
#define GC_NOALLOC_MAX_TILES 24576
#define GC_NOALLOC_DESC_BYTES (((GC_NOALLOC_MAX_GRIDS * sizeof(GcFusedGrid)) + 255) / 256 * 256)
#define GC_NOALLOC_SCRATCH_BYTES (GC_NOALLOC_DESC_BYTES + GC_NOALLOC_MAX_TILES * sizeof(int2))

/* the scratch: grid descriptors, then the tile work list */
static __device__ __align__(256) unsigned char g_noalloc_scratch[GC_NOALLOC_SCRATCH_BYTES];

int gc_default_variant();

namespace {

/* what one call sends to the GPU, by value in the launch parameters */
struct NoallocParams {
    int ngrids;
    int ntiles;
    int tile_start[GC_NOALLOC_MAX_GRIDS + 1]; /* first work-list entry of each grid */
    GcFusedGrid grids[GC_NOALLOC_MAX_GRIDS];
};
/* kernel parameters may take up to 32764 bytes (sm_70+, CUDA 12.1+) */
static_assert(sizeof(NoallocParams) <= 32000, "launch parameter block too large");

/* writes the descriptors and the (grid, tile) work list into the scratch */
__global__ void k_noalloc_fill(const __grid_constant__ NoallocParams p, GcFusedGrid *grids, int2 *tiles) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < p.ngrids) grids[t] = p.grids[t];
    if (t < p.ntiles) {
        int lo = 0, hi = p.ngrids - 1; /* the grid g with tile_start[g] <= t < tile_start[g+1] */
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.tile_start[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        tiles[t] = make_int2(lo, t - p.tile_start[lo]);
    }
}

constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_mu;

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

} // namespace

extern "C" int gcomcot_fused_step_noalloc(int ngrids, const gc_grid_step_io *grids, void *stream) {
    if (ngrids < 1 || !grids) {
        fprintf(stderr, "gcomcot_fused_step_noalloc: need at least one grid\n");
        return GC_EINVAL;
    }
    if (ngrids > GC_NOALLOC_MAX_GRIDS) {
        fprintf(stderr, "gcomcot_fused_step_noalloc: %d grids exceed the maximum of %d\n", ngrids,
                GC_NOALLOC_MAX_GRIDS);
        return GC_EINVAL;
    }
    for (int g = 0; g < ngrids; g++) {
        const gc_grid_step_io &q = grids[g];
        if (q.nx < 3 || q.ny < 3 || q.pitch < q.nx || (q.pitch % 32) != 0 || !q.z1 || !q.m1 || !q.n1 || !q.z2
            || !q.m2 || !q.n2 || !q.h || !q.rows) {
            fprintf(stderr, "gcomcot_fused_step_noalloc: grid %d: bad sizes or missing arrays "
                            "(nx,ny >= 3, pitch >= nx and a multiple of 32)\n", g);
            return GC_EINVAL;
        }
        if (!aligned16(q.z1) || !aligned16(q.m1) || !aligned16(q.n1) || !aligned16(q.z2) || !aligned16(q.m2)
            || !aligned16(q.n2) || !aligned16(q.h) || !aligned16(q.rows) || (q.zmax && !aligned16(q.zmax))) {
            fprintf(stderr, "gcomcot_fused_step_noalloc: grid %d: arrays must start on 16-byte boundaries\n", g);
            return GC_EINVAL;
        }
    }
    const int variant = gc_default_variant();
    int nxs[GC_NOALLOC_MAX_GRIDS], nys[GC_NOALLOC_MAX_GRIDS];
    for (int g = 0; g < ngrids; g++) { nxs[g] = grids[g].nx; nys[g] = grids[g].ny; }
    /* tile height: the engine's choice, raised until the work list fits */
    int ty = 0;
    long long ntiles = 0;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        int dev = 0;
        GC_CUDA_OR_RET(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices) return GC_ENOTSUP;
        if (!g_scratch_addr[dev]) {
            /* once per device, with that device current */
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr) {
                fprintf(stderr, "gcomcot_fused_step_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
                return GC_ECUDA;
            }
            g_scratch_addr[dev] = ptr;
        }
        ty = gc_fused_pick_ty(variant, ngrids, nxs, nys);
    }
    for (;; ty++) {
        ntiles = 0;
        for (int g = 0; g < ngrids; g++) ntiles += gc_fused_tiles(nxs[g], nys[g], ty, nullptr);
        if (ntiles <= GC_NOALLOC_MAX_TILES || ty >= 4096) break;
    }
    if (ntiles > GC_NOALLOC_MAX_TILES) {
        fprintf(stderr, "gcomcot_fused_step_noalloc: %lld tiles exceed the maximum of %d\n", ntiles,
                GC_NOALLOC_MAX_TILES);
        return GC_EINVAL;
    }
    NoallocParams p; /* on this thread's stack: the launch copies it */
    memset(&p, 0, sizeof p);
    p.ngrids = ngrids;
    int t = 0;
    for (int g = 0; g < ngrids; g++) {
        const gc_grid_step_io &q = grids[g];
        GcFusedGrid &d = p.grids[g];
        d.nx = q.nx; d.ny = q.ny; d.pitch = q.pitch; d.root = 1; d.explicit_r24 = 0;
        d.ty = ty;
        const int nt = gc_fused_tiles(q.nx, q.ny, ty, &d.tiles_x);
        /* step 1 of a one-step window: buffers [0] are read, [1] written */
        d.step0 = 1; d.cur0 = 0; d.nsteps = 1;
        d.flags = q.zmax ? GC_F_MAXAMP : 0;
        d.z[0] = const_cast<float *>(q.z1); d.z[1] = q.z2;
        d.m[0] = const_cast<float *>(q.m1); d.m[1] = q.m2;
        d.n[0] = const_cast<float *>(q.n1); d.n[1] = q.n2;
        d.h = q.h; d.rows = q.rows; d.zmax = q.zmax;
        p.tile_start[g] = t;
        t += nt;
    }
    p.tile_start[ngrids] = t;
    p.ntiles = t;
    int dev = 0;
    GC_CUDA_OR_RET(cudaGetDevice(&dev));
    cudaStream_t s = (cudaStream_t)stream;
    char *base = (char *)g_scratch_addr[dev];
    GcFusedGrid *d_grids = (GcFusedGrid *)base;
    int2 *d_tiles = (int2 *)(base + GC_NOALLOC_DESC_BYTES);
    GC_CUDA_OR_RET(gc_fused_clear_error_async(s));
    const int fill = t > ngrids ? t : ngrids;
    k_noalloc_fill<<<(fill + 255) / 256, 256, 0, s>>>(p, d_grids, d_tiles);
    GC_CUDA_OR_RET(cudaGetLastError());
    GC_CUDA_OR_RET(gc_fused_launch_multi(variant, d_grids, d_tiles, t, nullptr, 1, 0, s));
    return GC_OK;
}
