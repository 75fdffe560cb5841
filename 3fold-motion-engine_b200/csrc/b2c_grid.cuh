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
// every array of a grid present and its dims at least 8 per axis (the wrap-around query needs it)
inline bool grid_valid(const b2c_grid *g)
{
    return g && g->dim_x >= 8 && g->dim_y >= 8 && g->dim_z >= 8 && g->cell > 0.0f && g->bucket && g->start &&
           g->cursor && g->sorted && g->scan_tmp && g->sorted_pos;
}

// Visit every bead j > i of another body within (1e-9, 2R) of xi.  z is the innermost bucket
// coordinate, so each (x, y) column of the query block is one run of consecutive buckets, and
// its slots one range of `sorted`, unless the column wraps around the grid (then cell by cell).
// A candidate's id and its slot-ordered position and owner (spos) are independent loads.  The
// visiting order is not the bucket order; callers that emit in order sort by bead id.
template <class F>
__device__ __forceinline__ void visit_slots(int i, f3 xi, int bi, const float4 *__restrict__ spos,
                                            const int *__restrict__ sorted, int t0, int t1, F &&f)
{
    for (int t = t0; t < t1; ++t) {
        const int j = sorted[t];
        const float4 p = spos[t];
        if (j > i && __float_as_int(p.w) != bi) {
            const f3 xj = xyz(p);
            const f3 dvec = sub3(xi, xj);
            const float dist = len3(dvec);
            if (dist < B2C_2R && dist > 1e-9f) f(j, xj, dvec, dist);
        }
    }
}
template <class F>
__device__ __forceinline__ void for_each_bead_neighbor(int i, f3 xi, int bi, const float4 *__restrict__ spos,
                                                       const int *__restrict__ start, const int *__restrict__ sorted,
                                                       const GridView &g, F &&f)
{
    const QueryRange qr = query_range(xi, B2C_2R, g.inv);
    const int nz = qr.hi[2] - qr.lo[2];
    for (int iy = qr.lo[1]; iy <= qr.hi[1]; ++iy)
        for (int ix = qr.lo[0]; ix <= qr.hi[0]; ++ix) {
            const int b0 = bucket_of(g, ix, iy, qr.lo[2]), b1 = bucket_of(g, ix, iy, qr.hi[2]);
            if (b1 - b0 == nz) {
                visit_slots(i, xi, bi, spos, sorted, start[b0], start[b1 + 1], f);
            } else {
                for (int iz = qr.lo[2]; iz <= qr.hi[2]; ++iz) {
                    const int b = bucket_of(g, ix, iy, iz);
                    visit_slots(i, xi, bi, spos, sorted, start[b], start[b + 1], f);
                }
            }
        }
}

}  // namespace b2c
