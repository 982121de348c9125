// bvh_quant.hpp — 4-wide nodes with 8-bit child boxes (host and device).
//
// The 112-byte 4-wide node ({minx[4], maxx[4], miny[4], maxy[4], minz[4], maxz[4], refs[4]}, floats
// and int bits) is stored in 64 bytes after the compressed wide nodes of Ylitie, Karras and Laine
// ("Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017): per axis
// the node keeps an origin P (the smallest child minimum) and a power-of-two step 2^e, the least
// for which 255 steps span the node; each child plane is a byte q, the minimum rounded down and the
// maximum rounded up, so the box P + q * 2^e contains the child's box exactly (the differences
// are formed in double precision, where they are exact).  Words:
//   [0..2] P.x, P.y, P.z (float bits)   [3] (e.x + 127) | (e.y + 127) << 8 | (e.z + 127) << 16
//   [4] q min x  [5] q max x  [6] q min y  [7] q max y  [8] q min z  [9] q max z  (byte k: child k)
//   [10], [11] 0                         [12..15] child references (0x7fffffff: empty slot)
// Traversal only prunes with these boxes; which triangle a ray hits is decided by the exact test.
#pragma once

#include <cstdint>
#include <cstring>
#include <math.h>

#if defined(__CUDACC__)
#define PHX_QHD __host__ __device__ inline
#else
#define PHX_QHD inline
#endif

namespace phx {

constexpr int QNODE_WORDS = 16;
constexpr int32_t QNODE_EMPTY = 0x7fffffff;

PHX_QHD uint32_t qnode_f2u(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

// one 28-float 4-wide node -> 16 words
PHX_QHD void quantize_wide_node(const float *o, uint32_t *q) {
    int32_t refs[4];
    memcpy(refs, o + 24, 16);
    for (int w = 0; w < QNODE_WORDS; w++)
        q[w] = 0;
    uint32_t ebytes = 0;
    for (int a = 0; a < 3; a++) {
        float P = 1e30f, H = -1e30f;
        for (int k = 0; k < 4; k++)
            if (refs[k] != QNODE_EMPTY) {
                P = o[8 * a + k] < P ? o[8 * a + k] : P;
                H = o[8 * a + 4 + k] > H ? o[8 * a + 4 + k] : H;
            }
        if (!(P <= H)) { // no child (cannot happen: a node has at least two)
            P = 0.0f;
            H = 1.0f;
        }
        const double ext = (double)H - (double)P;
        int e = ext > 0.0 ? ilogb(ext) - 9 : -126;
        if (e < -126)
            e = -126;
        while (e < 127 && 255.0 * ldexp(1.0, e) < ext)
            e++;
        const double inv_step = ldexp(1.0, -e);
        uint32_t qlo = 0, qhi = 0;
        for (int k = 0; k < 4; k++) {
            uint32_t lo_b = 255, hi_b = 0;
            if (refs[k] != QNODE_EMPTY) {
                double l = floor(((double)o[8 * a + k] - (double)P) * inv_step);
                double h = ceil(((double)o[8 * a + 4 + k] - (double)P) * inv_step);
                l = l < 0.0 ? 0.0 : (l > 255.0 ? 255.0 : l);
                h = h < 0.0 ? 0.0 : (h > 255.0 ? 255.0 : h);
                lo_b = (uint32_t)l;
                hi_b = (uint32_t)h;
            }
            qlo |= lo_b << (8 * k);
            qhi |= hi_b << (8 * k);
        }
        q[a] = qnode_f2u(P);
        ebytes |= (uint32_t)(e + 127) << (8 * a);
        q[4 + 2 * a] = qlo;
        q[5 + 2 * a] = qhi;
    }
    q[3] = ebytes;
    memcpy(q + 12, refs, 16);
}

} // namespace phx
