/*
 * b2c -- B200-native rigid-body contact solve, C ABI.
 *
 * The drop-in boundary of the reference is the Python ContactEngine protocol
 * (src/motion_engine/contact_engine.py:48-55): step / get_state / set_kinematic /
 * contact_forces, implemented by RelaxedJacobiContactEngine
 * (src/motion_engine/contact_engine_gpu.py:191-299) and the coloured / ColorCache engines
 * (src/motion_engine/contact_engine_gpu_colored.py:793-1410,
 *  src/motion_engine/contact_engine_gpu_color_cache.py:21-54).  The reference has no
 * foreign-function interface for this path: its engines call Warp kernels (wp.launch)
 * directly.  The entry points below are what such an interface binds: one C function per
 * stage of a substep (each replaces the Warp launches named beside it), plus whole-substep
 * drivers.  The Python host package (3fold-motion-engine_b200/engine.py) implements the
 * ContactEngine protocol on top of them through ctypes.
 *
 * Conventions
 *  - Every pointer inside the structs is a DEVICE pointer allocated by the caller (PyTorch
 *    in the Python package).  The library never allocates or frees caller memory.
 *  - Vectors are float4 (x, y, z, pad) so every body / contact record is one 128-bit load.
 *  - Counts that the device produces (contacts, pairs, colours) stay on the device in a
 *    b2c_header; kernels read them there, so a whole step is a fixed launch sequence that
 *    can be captured into one CUDA graph with no host read-back in between.
 *  - Every call is asynchronous on the given stream and returns a status:
 *      0 OK, 1 bad argument, 2 capacity overflow (reported through the header),
 *      4 device wait timed out, 5 CUDA error.  b2c_last_error() gives the message.
 */
#ifndef B2C_H
#define B2C_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define B2C_API __attribute__((visibility("default")))
#else
#define B2C_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define B2C_OK 0
#define B2C_EARG 1
#define B2C_ECAPACITY 2
#define B2C_ETIMEOUT 4
#define B2C_ECUDA 5

/* error bits written by the kernels into b2c_header.error */
#define B2C_ERR_CONTACT_OVERFLOW 1   /* more contacts than b2c_contacts.capacity */
#define B2C_ERR_SEGMENT_OVERFLOW 2   /* a body pair with more than 1024 contacts (COL:669-674) */
#define B2C_ERR_CHUNK_OVERFLOW 4     /* a body pair with more than 8 kept contacts (COL:384-386) */
#define B2C_ERR_COLOR_OVERFLOW 8     /* more colours than the colour cap (COL:1199-1201) */
#define B2C_ERR_COLOR_TIMEOUT 16     /* colouring did not finish in its round budget (COL:1197) */
#define B2C_ERR_NEIGHBOR_OVERFLOW 32 /* a bead with more than 64 neighbours within 2R */
#define B2C_ERR_PAIR_OVERFLOW 64     /* more body pairs than the pair capacity */

typedef void *b2c_stream; /* a cudaStream_t */

/* Rigid bodies, structure of arrays.  Replaces the Warp arrays built in
 * RelaxedJacobiContactEngine._build (contact_engine_gpu.py:223-238). */
typedef struct b2c_bodies {
    int32_t n;
    float *xc;          /* (n,4) centre of mass */
    float *q;           /* (n,4) orientation quaternion (x, y, z, w) */
    float *v;           /* (n,4) linear velocity */
    float *w;           /* (n,4) angular velocity */
    float *pv;          /* (n,4) pseudo-velocity of the position pass */
    float *po;          /* (n,4) pseudo angular velocity of the position pass */
    float *invM;        /* (n) inverse mass, 0 for kinematic bodies */
    const float *IbInv; /* (n,12) body-frame inverse inertia, 3 rows padded to float4 */
    const int32_t *kin; /* (n) 1 = kinematic */
    float *invIw;       /* (n,12) world-frame inverse inertia rows, written each substep */
} b2c_bodies;

/* Bead clouds: the reference's voxelised boxes (_voxbox, contact_engine_gpu.py:186-188). */
typedef struct b2c_beads {
    int32_t n;              /* total beads over all bodies */
    const float *rest;      /* (n,4) bead offset in its body's frame */
    const int32_t *owner;   /* (n) body of each bead; beads of a body are contiguous */
    float *world;           /* (n,4) world position, written each substep */
} b2c_beads;

/* Uniform hash grid over the beads (the reference uses wp.HashGrid, built at
 * contact_engine_gpu.py:262).  Cell coordinates wrap modulo the dims, so a query's
 * 3x3x3 block never aliases onto itself as long as every dim is >= 8. */
typedef struct b2c_grid {
    int32_t dim_x, dim_y, dim_z;
    float cell;         /* cell edge = contact distance 2R */
    int32_t *bucket;    /* (beads) bucket of each bead */
    int32_t *start;     /* (dims+1) first slot of each bucket in `sorted` */
    int32_t *cursor;    /* (dims+1) bucket counts, then scatter cursors */
    int32_t *sorted;    /* (beads) bead ids grouped by bucket */
    int32_t *scan_tmp;  /* scan scratch, b2c_scan_scratch_ints(dims+1) ints */
} b2c_grid;

/* Contacts, structure of arrays of float4 records. */
typedef struct b2c_contacts {
    int32_t capacity;
    int32_t *bi, *bj;   /* body A, body B (-1 = ground) */
    float *pA;          /* (cap,4) point on A, .w = penetration depth */
    float *pB;          /* (cap,4) point on B */
    float *n;           /* (cap,4) contact normal, pointing from B to A */
    int32_t *fa, *fb;   /* feature ids: bead of A, bead of B or -1 */
    float *imp;         /* (cap,4) accumulated impulses jn, jt1, jt2, jp */
} b2c_contacts;

/* Device-resident per-substep counters (read once per step by the host, after the fact). */
typedef struct b2c_header {
    int32_t n_raw;       /* contacts generated (may exceed capacity) */
    int32_t n_contacts;  /* contacts stored */
    int32_t n_kept;      /* after manifold reduction */
    int32_t n_pairs;     /* body pairs */
    int32_t n_colors;    /* colours of the pair graph */
    int32_t cache_hit;   /* 1 when the colour cache was reused this substep */
    int32_t error;       /* B2C_ERR_* bits, sticky until cleared by the host */
    int32_t rounds;      /* Jones-Plassmann rounds of the last colouring */
} b2c_header;

/* Relaxed-Jacobi parameters (RelaxedJacobiContactEngine.__init__, contact_engine_gpu.py:195). */
typedef struct b2c_jacobi_params {
    int32_t vit, pit;
    float relax, mu;
} b2c_jacobi_params;

/* ---- version / errors ---- */
B2C_API int32_t b2c_version(void);
B2C_API const char *b2c_last_error(void);
/* ints of scratch that b2c_exclusive_scan needs for n elements */
B2C_API int32_t b2c_scan_scratch_ints(int32_t n);
/* exclusive prefix sum of n int32 (device pointers); out may alias nothing */
B2C_API int32_t b2c_exclusive_scan(const int32_t *in, int32_t *out, int32_t n, int32_t *scratch, b2c_stream s);

/* ---- per-body stages ---- */
/* k_grav + k_invIw (contact_engine_gpu.py:40-53): v += g dt for dynamic bodies;
 * invIw = R IbInv R^T (zero when kinematic). */
B2C_API int32_t b2c_body_predict(const b2c_bodies *b, float dt, b2c_stream s);
/* k_integ (contact_engine_gpu.py:171-180): x += (v+pv) dt; q <- normalize(q + 0.5 (w+po) q dt). */
B2C_API int32_t b2c_body_integrate(const b2c_bodies *b, float dt, b2c_stream s);

/* ---- bead broadphase and narrowphase ---- */
/* k_worldp (contact_engine_gpu.py:55-59) + bucket of each bead. */
B2C_API int32_t b2c_bead_world(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, b2c_stream s);
/* HashGrid.build (contact_engine_gpu.py:262): counting sort of the beads by bucket. */
B2C_API int32_t b2c_grid_build(const b2c_beads *beads, b2c_grid *g, b2c_stream s);
/* k_gen / k_gen_fid (contact_engine_gpu.py:61-79, contact_engine_gpu_colored.py:102-122):
 * ground contacts and bead-bead contacts closer than 2R, appended in arbitrary order
 * (the Jacobi sum is order free).  Resets hdr->n_raw / n_contacts first. */
B2C_API int32_t b2c_bead_contacts(const b2c_beads *beads, const b2c_grid *g, b2c_contacts *c, b2c_header *hdr,
                          b2c_stream s);

/* ---- relaxed Jacobi solve (contact_engine_gpu.py:266-275) ---- */
/* acc: (6, bodies) int64 fixed-point accumulators, zero on entry and on return.
 * Zeroes the impulses and pv/po (only when there are contacts, as the reference does),
 * then vit x (k_jac_vel, k_apply) and pit x (k_jac_pos, k_apply). */
B2C_API int32_t b2c_jacobi_solve(const b2c_bodies *b, b2c_contacts *c, const b2c_header *hdr, int64_t *acc,
                         const b2c_jacobi_params *p, float dt, b2c_stream s);

/* One whole relaxed-Jacobi substep: predict, bead world, grid, contacts, solve, integrate.
 * vgrav (n,4) receives the velocity after gravity (the contact-force reference point of
 * contact_engine_gpu.py:265,279). */
B2C_API int32_t b2c_jacobi_substep(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, b2c_contacts *c,
                           b2c_header *hdr, int64_t *acc, const b2c_jacobi_params *p, float dt, float *vgrav,
                           b2c_stream s);

#ifdef __cplusplus
}
#endif
#endif /* B2C_H */
