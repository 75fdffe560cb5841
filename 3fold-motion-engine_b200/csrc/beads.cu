// Bead clouds: world positions, uniform hash grid, contact generation.
#include "b2c_grid.cuh"

namespace b2c {

int exclusive_scan(const int *in, int *out, int n, const int *dn, int *scratch, cudaStream_t s);

// k_worldp, contact_engine_gpu.py:55-59: allp = xc[b] + quat_rotate(q[b], rest)
__global__ void k_bead_world(int nb, const float *__restrict__ xc, const float *__restrict__ q,
                             const float *__restrict__ rest, const int *__restrict__ owner, float *__restrict__ world,
                             int *__restrict__ bucket, GridView g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const int b = owner[i];
    f3 p = add3(ld3(xc, b), quat_rotate(ldq(q, b), ld3(rest, i)));
    st4(world, i, f4(p, 0.0f));
    bucket[i] = bucket_of(g, cellc(p.x, g.inv), cellc(p.y, g.inv), cellc(p.z, g.inv));
}

__global__ void k_grid_count(int nb, const int *__restrict__ bucket, int *__restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) atomicAdd(count + bucket[i], 1);
}

// slot of bead i in its bucket; the slot also receives the bead's position and owner
__global__ void k_grid_scatter(int nb, const int *__restrict__ bucket, const int *__restrict__ start,
                               int *__restrict__ cursor, int *__restrict__ sorted, const float *__restrict__ world,
                               const int *__restrict__ owner, float4 *__restrict__ spos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const int b = bucket[i];
    const int t = start[b] + atomicAdd(cursor + b, 1);
    sorted[t] = i;
    spos[t] = f4(ld3(world, i), __int_as_float(owner[i]));
}

__device__ __forceinline__ void append_contact(b2c_contacts c, int *n_raw, int bi, int bj, f3 pA, f3 pB, f3 nrm,
                                               float pen, int fa, int fb)
{
    const int k = atomicAdd(n_raw, 1);
    if (k >= c.capacity) return;
    c.bi[k] = bi;
    c.bj[k] = bj;
    st4(c.pA, k, f4(pA, pen));
    st4(c.pB, k, f4(pB, 0.0f));
    st4(c.n, k, f4(nrm, 0.0f));
    c.fa[k] = fa;
    c.fb[k] = fb;
}

// k_gen / k_gen_fid, contact_engine_gpu.py:61-79 and contact_engine_gpu_colored.py:102-122.
// Ground: z - R < 0 -> normal +z, depth R - z.  Bead pairs: j > i, other body,
// 1e-9 < |xi - xj| < 2R -> normal (xi - xj)/dist, depth 2R - dist, body A owns bead i.
__global__ void k_bead_contacts(int nb, const float *__restrict__ world, const int *__restrict__ owner,
                                const int *__restrict__ start, const int *__restrict__ sorted,
                                const float4 *__restrict__ spos, GridView g, b2c_contacts c, b2c_header *hdr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const f3 xi = ld3(world, i);
    const int bi = owner[i];
    const float s = xi.z - B2C_R;
    if (s < 0.0f) append_contact(c, &hdr->n_raw, bi, -1, xi, f3{0.0f, 0.0f, 0.0f}, f3{0.0f, 0.0f, 1.0f}, -s, i, -1);
    for_each_bead_neighbor(i, xi, bi, spos, start, sorted, g, [&](int j, f3 xj, f3 dvec, float dist) {
        append_contact(c, &hdr->n_raw, bi, owner[j], xi, xj, div3(dvec, dist), B2C_2R - dist, i, j);
    });
}

__global__ void k_header_reset_contacts(b2c_header *hdr)
{
    hdr->n_raw = 0;
    hdr->n_contacts = 0;
}

__global__ void k_header_finish_contacts(b2c_header *hdr, int cap)
{
    const int raw = hdr->n_raw;
    hdr->n_contacts = raw < cap ? raw : cap;
    if (raw > cap) hdr->error |= B2C_ERR_CONTACT_OVERFLOW;
}


int bead_world(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, cudaStream_t s)
{
    if (beads->n <= 0) return B2C_OK;
    k_bead_world<<<blocks_for(beads->n), kThreads, 0, s>>>(beads->n, b->xc, b->q, beads->rest, beads->owner,
                                                           beads->world, g->bucket, view_of(g));
    return check_launch("bead_world");
}

int grid_build(const b2c_beads *beads, b2c_grid *g, cudaStream_t s)
{
    const int nbk = g->dim_x * g->dim_y * g->dim_z;
    cudaMemsetAsync(g->cursor, 0, sizeof(int) * (size_t)(nbk + 1), s);
    if (beads->n > 0) k_grid_count<<<blocks_for(beads->n), kThreads, 0, s>>>(beads->n, g->bucket, g->cursor);
    int rc = check_launch("grid_count");
    if (rc) return rc;
    // start[] over nbk+1 entries: the extra trailing count reads as zero and start[nbk] = beads
    rc = exclusive_scan(g->cursor, g->start, nbk + 1, nullptr, g->scan_tmp, s);
    if (rc) return rc;
    cudaMemsetAsync(g->cursor, 0, sizeof(int) * (size_t)nbk, s);
    if (beads->n > 0)
        k_grid_scatter<<<blocks_for(beads->n), kThreads, 0, s>>>(beads->n, g->bucket, g->start, g->cursor, g->sorted,
                                                                 beads->world, beads->owner,
                                                                 reinterpret_cast<float4 *>(g->sorted_pos));
    return check_launch("grid_scatter");
}

int bead_contacts(const b2c_beads *beads, const b2c_grid *g, b2c_contacts *c, b2c_header *hdr, cudaStream_t s)
{
    k_header_reset_contacts<<<1, 1, 0, s>>>(hdr);
    if (beads->n > 0)
        k_bead_contacts<<<blocks_for(beads->n, 128), 128, 0, s>>>(
            beads->n, beads->world, beads->owner, g->start, g->sorted,
            reinterpret_cast<const float4 *>(g->sorted_pos), view_of(g), *c, hdr);
    k_header_finish_contacts<<<1, 1, 0, s>>>(hdr, c->capacity);
    return check_launch("bead_contacts");
}

}  // namespace b2c

static bool grid_ok(const b2c_grid *g) { return b2c::grid_valid(g); }

extern "C" int32_t b2c_bead_world(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, b2c_stream s)
{
    if (!b || !beads || !grid_ok(g) || beads->n < 0 || (beads->n > 0 && (!beads->rest || !beads->owner || !beads->world))) {
        b2c::set_error("b2c_bead_world: bad argument");
        return B2C_EARG;
    }
    return b2c::bead_world(b, beads, g, b2c::stream_of(s));
}

extern "C" int32_t b2c_grid_build(const b2c_beads *beads, b2c_grid *g, b2c_stream s)
{
    if (!beads || !grid_ok(g)) {
        b2c::set_error("b2c_grid_build: bad argument");
        return B2C_EARG;
    }
    return b2c::grid_build(beads, g, b2c::stream_of(s));
}

extern "C" int32_t b2c_bead_contacts(const b2c_beads *beads, const b2c_grid *g, b2c_contacts *c, b2c_header *hdr,
                                     b2c_stream s)
{
    if (!beads || !grid_ok(g) || !c || !hdr || c->capacity < 0) {
        b2c::set_error("b2c_bead_contacts: bad argument");
        return B2C_EARG;
    }
    return b2c::bead_contacts(beads, g, c, hdr, b2c::stream_of(s));
}
