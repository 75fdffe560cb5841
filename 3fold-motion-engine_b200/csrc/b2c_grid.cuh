// Uniform hash-grid helpers shared by the bead kernels.  Cell coordinates wrap modulo the
// grid dims, so the at most 4x4x4 cells of one query never alias onto each other (dims >= 8).
#pragma once
#include "b2c_common.cuh"

namespace b2c {

struct GridView {
    int dx, dy, dz;
    float inv;  // 1 / cell
};

__device__ __forceinline__ int wrapi(int a, int m)
{
    int r = a % m;
    return r < 0 ? r + m : r;
}
__device__ __forceinline__ int cellc(float x, float inv) { return (int)floorf(x * inv); }
__device__ __forceinline__ int bucket_of(const GridView &g, int ix, int iy, int iz)
{
    return (wrapi(ix, g.dx) * g.dy + wrapi(iy, g.dy)) * g.dz + wrapi(iz, g.dz);
}

// Query block of a point: every cell within 2R plus a 1 % margin, so a neighbour at a cell
// boundary is never missed by rounding; the exact distance test of the caller decides.
struct QueryRange {
    int lo[3], hi[3];
};
__device__ __forceinline__ QueryRange query_range(f3 p, float r, float inv)
{
    const float m = r * 1.01f;
    QueryRange q;
    q.lo[0] = cellc(p.x - m, inv);
    q.hi[0] = cellc(p.x + m, inv);
    q.lo[1] = cellc(p.y - m, inv);
    q.hi[1] = cellc(p.y + m, inv);
    q.lo[2] = cellc(p.z - m, inv);
    q.hi[2] = cellc(p.z + m, inv);
    return q;
}

inline GridView view_of(const b2c_grid *g) { return GridView{g->dim_x, g->dim_y, g->dim_z, 1.0f / g->cell}; }

// Visit every bead j > i of another body within (1e-9, 2R) of xi, in bucket order.
template <class F>
__device__ __forceinline__ void for_each_bead_neighbor(int i, f3 xi, int bi, const float *__restrict__ world,
                                                       const int *__restrict__ owner, const int *__restrict__ start,
                                                       const int *__restrict__ sorted, const GridView &g, F &&f)
{
    const QueryRange qr = query_range(xi, B2C_2R, g.inv);
    for (int iz = qr.lo[2]; iz <= qr.hi[2]; ++iz)
        for (int iy = qr.lo[1]; iy <= qr.hi[1]; ++iy)
            for (int ix = qr.lo[0]; ix <= qr.hi[0]; ++ix) {
                const int b = bucket_of(g, ix, iy, iz);
                const int e = start[b + 1];
                for (int t = start[b]; t < e; ++t) {
                    const int j = sorted[t];
                    if (j > i && owner[j] != bi) {
                        const f3 xj = ld3(world, j);
                        const f3 dvec = sub3(xi, xj);
                        const float dist = len3(dvec);
                        if (dist < B2C_2R && dist > 1e-9f) f(j, xj, dvec, dist);
                    }
                }
            }
}

}  // namespace b2c
