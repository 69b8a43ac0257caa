// y-slab halos: the rows a slab sends to, and receives from, the slabs above and below it.
//
// A slab context holds the rows of its own slab plus `halo` rows on each side, every one of
// the M x 9 population planes laid out [member][q][y][x] as in a whole-grid context.  After k
// steps the outer 2k rows on each side are stale; the neighbours own those rows and send them.
// The packed form of `rows` rows is [plane][rows][nx], one buffer per neighbour, so one
// transfer per neighbour carries every member and direction.  This replaces the reference's
// member-sharded layout, whose analysis needs an all-to-all transpose per cycle
// (src/util/letkf_solver.h:135-215, 374-394; src/letkf.cu:191, 273, 315).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "lbl_internal.h"

namespace lbl {
namespace {

// grid (x: 16-byte words of one plane's rows, y: plane, z: 0 = the previous slab's rows, 1 = the next's)
__global__ void __launch_bounds__(256) slab_halo_kernel(uint4* __restrict__ f, int row_words, int ny, int rows,
                                                        int a_prev, int a_next, uint4* __restrict__ buf_prev,
                                                        uint4* __restrict__ buf_next, bool unpack) {
    const int plane = blockIdx.y;
    const bool next = blockIdx.z != 0;
    const int a = next ? a_next : a_prev;
    const size_t seg = size_t(rows) * row_words;
    uint4* buf = (next ? buf_next : buf_prev) + size_t(plane) * seg;
    uint4* g = f + (size_t(plane) * ny + a) * row_words;
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < seg; e += size_t(gridDim.x) * blockDim.x) {
        if (unpack)
            g[e] = buf[e];
        else
            buf[e] = g[e];
    }
}

}  // namespace

void launch_slab_halo(void* f, size_t elem, int nx, int ny, int planes, int rows, int a_prev, int a_next,
                      void* buf_prev, void* buf_next, bool unpack, cudaStream_t s) {
    const int row_words = int(size_t(nx) * elem / sizeof(uint4));
    const long long seg = (long long)rows * row_words;
    const int bx = int(std::min<long long>((seg + 255) / 256, 8));
    slab_halo_kernel<<<dim3(bx, planes, 2), 256, 0, s>>>(static_cast<uint4*>(f), row_words, ny, rows, a_prev, a_next,
                                                         static_cast<uint4*>(buf_prev), static_cast<uint4*>(buf_next),
                                                         unpack);
}

}  // namespace lbl
