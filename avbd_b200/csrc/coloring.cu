// coloring.cu -- exact DSATUR graph coloring on the GPU.
//
// ColorList::greedyColor2 (common/ColorList.hpp:149-241) colors one vertex per
// round: the uncolored vertex with the largest saturation (number of distinct
// colors among its colored neighbours), ties to the larger degree, then to
// the lower index, receives the smallest color unused by its neighbours.  The
// coloring fixes the Gauss-Seidel order of the solve, so it must be identical,
// not merely valid.
//
// One CTA colors one scene.  Every round is a block-wide arg-max over the
// packed key (saturation, degree, ~index) followed by the color choice and the
// saturation update of the winner's neighbours by one warp.  Per-vertex state
// (saturation and color, 2 bytes each) lives in shared memory when the scene
// fits, otherwise in a global scratch array.  Scenes are disjoint components,
// and DSATUR restricted to one component makes the same picks in the same
// relative order as DSATUR over the whole graph, so per-scene coloring equals
// the reference's coloring of the combined context.
#include "engine.h"

namespace avbd {

static constexpr int DS_THREADS = 512;
static constexpr unsigned short UNCOLORED = 0xFFFFu;

__global__ void __launch_bounds__(DS_THREADS) k_dsatur(const uint32_t* __restrict__ p_off,
                                                       const uint32_t* __restrict__ p_nbr,
                                                       const uint32_t* __restrict__ scene_begin,
                                                       uint32_t* __restrict__ color_out,
                                                       uint32_t* __restrict__ scene_ncolors,
                                                       unsigned short* __restrict__ g_scratch,
                                                       unsigned smem_vertices, int* __restrict__ error) {
    extern __shared__ unsigned char smem[];
    __shared__ unsigned long long warp_best[DS_THREADS / 32];
    __shared__ unsigned long long best_key;
    __shared__ uint32_t used[8];
    __shared__ unsigned max_color;

    const unsigned s = blockIdx.x;
    const unsigned v0 = scene_begin[s], v1 = scene_begin[s + 1];
    const unsigned n = v1 - v0;
    unsigned short* sat;
    unsigned short* col;
    if (n <= smem_vertices) {
        sat = reinterpret_cast<unsigned short*>(smem);
        col = sat + n;
    } else {
        sat = g_scratch + 2ull * v0;
        col = sat + n;
    }
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
        sat[i] = 0;
        col[i] = UNCOLORED;
    }
    if (threadIdx.x == 0) max_color = 0;
    __syncthreads();

    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (unsigned round = 0; round < n; round++) {
        // arg-max of (saturation, degree, lowest index) over uncolored vertices
        unsigned long long kmax = 0;
        for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
            if (col[i] != UNCOLORED) continue;
            unsigned deg = p_off[v0 + i + 1] - p_off[v0 + i];
            unsigned long long key = ((unsigned long long)sat[i] << 48) | ((unsigned long long)(deg & 0xFFFFu) << 32) |
                                     (unsigned long long)(0xFFFFFFFFu - i);
            kmax = key > kmax ? key : kmax;
        }
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) {
            unsigned long long o = __shfl_xor_sync(0xffffffffu, kmax, m);
            kmax = o > kmax ? o : kmax;
        }
        if (lane == 0) warp_best[warp] = kmax;
        __syncthreads();
        if (warp == 0) {
            unsigned long long k = lane < DS_THREADS / 32 ? warp_best[lane] : 0ull;
#pragma unroll
            for (int m = 16; m >= 1; m >>= 1) {
                unsigned long long o = __shfl_xor_sync(0xffffffffu, k, m);
                k = o > k ? o : k;
            }
            // winner: color = smallest color unused by its neighbours
            const unsigned v = 0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFull);
            const unsigned b = p_off[v0 + v], e = p_off[v0 + v + 1];
            if (lane < 8) used[lane] = 0;
            __syncwarp();
            for (unsigned t = b + lane; t < e; t += 32) {
                unsigned w = p_nbr[t] - v0;
                unsigned short cw = col[w];
                if (cw != UNCOLORED && cw < 256) atomicOr(&used[cw >> 5], 1u << (cw & 31));
            }
            __syncwarp();
            unsigned c = 0xFFFFFFFFu;
            if (lane < 8) {
                uint32_t freebits = ~used[lane];
                if (freebits) c = lane * 32 + __ffs(freebits) - 1;
            }
#pragma unroll
            for (int m = 16; m >= 1; m >>= 1) {
                unsigned o = __shfl_xor_sync(0xffffffffu, c, m);
                c = o < c ? o : c;
            }
            if (c >= 256) {
                if (lane == 0) atomicExch(error, AVBD_ERR_COLORS);
                c = 255;
            }
            if (lane == 0) {
                col[v] = (unsigned short)c;
                if (c + 1 > max_color) max_color = c + 1;
            }
            __syncwarp();
            // saturation update: c is new for an uncolored neighbour u unless
            // another colored neighbour of u already has it
            for (unsigned t = b + lane; t < e; t += 32) {
                unsigned u = p_nbr[t] - v0;
                if (col[u] != UNCOLORED) continue;
                bool seen = false;
                for (unsigned q = p_off[v0 + u]; q < p_off[v0 + u + 1]; q++) {
                    unsigned w = p_nbr[q] - v0;
                    if (w != v && col[w] == c) { seen = true; break; }
                }
                if (!seen) sat[u] = sat[u] + 1;
            }
        }
        __syncthreads();
    }
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) color_out[v0 + i] = col[i];
    if (threadIdx.x == 0) scene_ncolors[s] = max_color;
}

#define CK(x)                                                      \
    do {                                                           \
        cudaError_t e_ = (x);                                      \
        if (e_ != cudaSuccess) {                                   \
            err = std::string(#x) + ": " + cudaGetErrorString(e_); \
            goto fail;                                             \
        }                                                          \
    } while (0)

int gpu_dsatur(const std::vector<unsigned>& p_off, const std::vector<unsigned>& p_nbr,
               const std::vector<unsigned>& scene_begin, std::vector<unsigned>& color, unsigned& num_colors,
               cudaStream_t st, std::string& err) {
    const unsigned n = (unsigned)p_off.size() - 1;
    const unsigned ns = (unsigned)scene_begin.size() - 1;
    uint32_t *d_off = nullptr, *d_nbr = nullptr, *d_sb = nullptr, *d_col = nullptr, *d_nc = nullptr;
    unsigned short* d_scr = nullptr;
    int* d_err = nullptr;
    int herr = 0;
    std::vector<uint32_t> nc(ns, 0);
    int rc = AVBD_ERR_CUDA;
    unsigned max_scene = 0;
    for (unsigned s = 0; s < ns; s++) max_scene = std::max(max_scene, scene_begin[s + 1] - scene_begin[s]);
    // shared memory: 4 bytes per vertex, up to 200 KB
    const unsigned smem_limit = 200u * 1024u;
    unsigned smem_vertices = smem_limit / 4;
    size_t smem = std::min<size_t>((size_t)max_scene * 4, smem_limit);
    color.assign(n, 0);
    num_colors = 0;
    if (n == 0) return AVBD_OK;
    CK(cudaMalloc(&d_off, sizeof(uint32_t) * (n + 1)));
    CK(cudaMalloc(&d_nbr, sizeof(uint32_t) * std::max<size_t>(p_nbr.size(), 1)));
    CK(cudaMalloc(&d_sb, sizeof(uint32_t) * (ns + 1)));
    CK(cudaMalloc(&d_col, sizeof(uint32_t) * n));
    CK(cudaMalloc(&d_nc, sizeof(uint32_t) * ns));
    CK(cudaMalloc(&d_err, sizeof(int)));
    if (max_scene > smem_vertices) CK(cudaMalloc(&d_scr, sizeof(unsigned short) * 2 * (size_t)n));
    CK(cudaMemcpyAsync(d_off, p_off.data(), sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice, st));
    if (!p_nbr.empty())
        CK(cudaMemcpyAsync(d_nbr, p_nbr.data(), sizeof(uint32_t) * p_nbr.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_sb, scene_begin.data(), sizeof(uint32_t) * (ns + 1), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    CK(cudaFuncSetAttribute(k_dsatur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_dsatur<<<ns, DS_THREADS, smem, st>>>(d_off, d_nbr, d_sb, d_col, d_nc, d_scr, smem_vertices, d_err);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(color.data(), d_col, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(nc.data(), d_nc, sizeof(uint32_t) * ns, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (unsigned s = 0; s < ns; s++) num_colors = std::max(num_colors, nc[s]);
    if (herr) {
        err = "Ran out of colors (more than 256)";
        rc = herr;
    } else {
        rc = AVBD_OK;
    }
fail:
    cudaFree(d_off);
    cudaFree(d_nbr);
    cudaFree(d_sb);
    cudaFree(d_col);
    cudaFree(d_nc);
    cudaFree(d_err);
    cudaFree(d_scr);
    return rc;
}

}  // namespace avbd
