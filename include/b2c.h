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
    const int32_t *bead_start; /* (bodies+1) first bead of each body */
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
    float *sorted_pos;  /* (beads x 4) per slot of `sorted`: the bead's world position and, as the
                           bit pattern of .w, its owner body (written by b2c_grid_build) */
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

#define B2C_ERR_BARRIER_TIMEOUT 128  /* a grid barrier of the persistent solve gave up waiting */

/* uint32 words of a grid-barrier buffer (b2c_pairs.barrier, b2c_ncp_state.barrier): the arrival
 * counter, alone on its 128-byte line; b2c_barrier_words() returns it */
#define B2C_BARRIER_WORDS 32

/* Scratch of the coloured chain's ordering and manifold stage (one slot per raw contact
 * unless noted).  Replaces the radix-sort buffers, segment flags and selection arrays of
 * _device_manifold (contact_engine_gpu_colored.py:1050-1087). */
typedef struct b2c_manifold {
    int32_t capacity;        /* raw contacts */
    int32_t pair_capacity;   /* body pairs */
    int32_t *bead_count;     /* (beads+1) contacts emitted per bead */
    int32_t *bead_offset;    /* (beads+1) exclusive scan of bead_count: feature-order offsets */
    int32_t *pair_local;     /* rank of the contact's pair among its body's pairs */
    int32_t *pair_first;     /* first-occurrence start / count of a pair (packed 2 ints per slot) */
    int32_t *gorder;         /* pair-sorted position -> feature index */
    int32_t *body_npairs;    /* (bodies+1) pairs per body */
    int32_t *pair_base;      /* (bodies+1) exclusive scan of body_npairs */
    int32_t *praw_start;     /* (pair_capacity) first pair-sorted position of each pair */
    int32_t *praw_count;     /* (pair_capacity) raw contacts of each pair */
    double *jn_in;           /* warm-started normal impulse (float64, as COL:604) */
    double *jn_red;          /* normal impulse after redistribution onto the kept points */
    float *jt_in;            /* (cap,2) warm-started friction impulses */
    int32_t *keep;           /* 1 = kept by the selection */
    int32_t *kidx;           /* exclusive scan of keep: kept index */
    int32_t *scan_tmp;       /* b2c_scan_scratch_ints(max(beads+1, capacity+1, pairs+1)) */
} b2c_manifold;

/* Kept contacts and their body pairs, the colouring, the colour cache and the warm store. */
typedef struct b2c_pairs {
    int32_t capacity;        /* pairs */
    int32_t max_colors;      /* capacity of the per-colour arrays (the reference's _NCOLMAX = 512) */
    int32_t *pbi, *pbj;      /* bodies of each pair, sorted by (pbi, pbj) */
    int32_t *kcount;         /* kept contacts of each pair */
    int32_t *pstart;         /* exclusive scan of kcount */
    int32_t *pidx;           /* (kept cap) kept-contact index, pair-sorted, feature order inside a pair */
    int32_t *col;            /* colour of each pair */
    int32_t *porder;         /* pairs grouped by colour */
    int32_t *cstart, *ccount;/* (max_colors) per-colour offset and count into porder */
    int64_t *claim;          /* (2 x bodies) Jones-Plassmann claims, two alternating arrays */
    int32_t *cached_a, *cached_b; /* colour cache: pbi / pbj of the cached colouring */
    float *cached_mass;      /* (bodies) invM of the cached colouring */
    int32_t *cache_state;    /* [cached pair count, cached colour count, valid, hits, misses] */
    uint32_t *barrier;       /* (B2C_BARRIER_WORDS) the persistent solve's grid barrier: its arrival
                                counter, cleared before each cooperative launch */
    float *rec;              /* colour-major pair records of the solve, b2c_pair_record_floats()
                                floats: per slot a header, both bodies' inverse inertia and mass,
                                and per contact its normal|depth, the terms that stay fixed
                                during a solve (rA|meff, rB|meft1, t1|meft2) and its impulses.
                                The colouring uses the header words as scratch. */
    int32_t kslots;          /* contact slots per record (>= the most contacts one pair keeps) */
    uint64_t *body_colors;   /* (bodies) colours used around each body; needed with
                                B2C_COLOR_FIRST_FIT only, else NULL */
    const int32_t *body_local; /* (bodies) index of each body inside its scene, or NULL.  Set:
                                the colouring priority hashes the pair's scene-local bodies
                                (a scene colours alike alone or in a batch); NULL: the
                                reference's hash of the pair index (COL:136-148). */
    int32_t *body_slots;     /* (bodies x 64) or NULL.  With B2C_COLOR_FIRST_FIT, B2C_COLOR_ROW_FORM
                                and B2C_COLOR_APPLY_WARM the solve's record gather writes, for
                                each dynamic body b and colour c of one of its pairs, that
                                pair's record slot x 2 + side (0: body A, 1: body B) at
                                [64 b + c]; the warm start is then applied body by body in
                                colour order (the same bits as colour by colour) instead of in
                                one pass of colour phases. */
    /* Scene schedule of the solve (b2c_color_params.solve_blocks == B2C_SOLVE_SCENES, row form):
     * one CTA per scene, each scene's colour phases separated by its own CTA barrier, not by
     * a barrier over all scenes.  Scenes share no bodies, so the bits are those of the other
     * forms.  The bodies of a scene are contiguous and the scenes in body order; a scene's pairs
     * are then contiguous too (pairs are sorted by their first body).  Zero / NULL when unused. */
    int32_t n_scenes;
    const int32_t *scene_body_start; /* (n_scenes+1) first body of each scene */
    const int32_t *scene_order;      /* (n_scenes) launch order of the scenes (largest first), or NULL */
    int32_t *pair_slot;              /* (capacity) record slot of each pair, written by the gather */
    int32_t *scene_slots;            /* (capacity) each scene's record slots grouped by colour */
    int32_t *prio_hi;                /* (capacity) or NULL: with B2C_COLOR_REDUCED_CONTACTS the
                                        high part of each chunk's colouring priority (slot << 19 |
                                        run parity << 18), written by b2c_manifold_reduce */
    int32_t *isl_work;               /* b2c_island_work_ints(bodies, capacity) ints, zero-filled
                                        before the first substep, or NULL: the island partition of
                                        the solve with B2C_COLOR_ISLANDS */
} b2c_pairs;

/* Warm-start store: kept feature keys (sorted) and their impulses, from the previous substep. */
typedef struct b2c_warm {
    int32_t capacity;
    int64_t *keys;           /* (cap) */
    float *imp;              /* (cap,4) jn, jt1, jt2, unused */
    int32_t *n;              /* (1) entries stored */
} b2c_warm;

/* Boxes for the box/plane + box/box narrowphase (ncp/ncp_gpu.py:1097-1227): per-body half
 * extents, a body-AABB hash grid, candidate pairs and per-candidate contact slots. */
typedef struct b2c_boxes {
    int32_t n;
    const float *half;        /* (n,4) half extents */
    const float *mu;          /* (n) friction per body (contact: sqrt(mu_a mu_b), ground: mu_a) or NULL */
    float margin;             /* contact margin (the reference's 2e-3) */
    float cell;               /* broadphase cell >= 2 x the largest AABB half extent + margin */
    int32_t dim_x, dim_y, dim_z; /* broadphase hash-grid dims (>= 8 each) */
    int32_t cand_capacity;    /* candidate pairs (ground + box-box) */
    int32_t *bucket;          /* (n) */
    int32_t *start;           /* (dims+1) */
    int32_t *cursor;          /* (dims+1) */
    int32_t *sorted;          /* (n) */
    int32_t *cand_count;      /* (n+1) candidates owned by each body */
    int32_t *cand_offset;     /* (n+1) */
    int32_t *cand_a, *cand_b; /* (cand cap) candidate pair, b = -1 for the ground */
    int32_t *cont_count;      /* (cand cap+1) contacts of each candidate */
    int32_t *cont_offset;     /* (cand cap+1) */
    int32_t *pair_flag;       /* (cand cap+1) 1 when the candidate has contacts */
    int32_t *pair_offset;     /* (cand cap+1) */
    float *slot_p;            /* (cand cap x 8, 4) contact point | gap */
    float *slot_n;            /* (cand cap, 4) normal from b to a */
    int32_t *slot_f;          /* (cand cap x 8) feature id */
    int32_t *scan_tmp;        /* b2c_scan_scratch_ints(max(dims, n, cand cap) + 1) */
    const int32_t *scene;     /* (n) scene of each body for a batch of independent scenes, or
                                 NULL (one scene).  Bodies of different scenes never pair; the
                                 scenes may overlap in space (the grid hash includes the scene). */
} b2c_boxes;

/* Flags of b2c_color_params.flags */
#define B2C_COLOR_FIXED_FRAME 1  /* normal-derived tangent frame (contact_engine_gpu_fixed_frame.py) */
#define B2C_COLOR_APPLY_WARM 2   /* apply the warm impulses once per colour before the sweeps */
#define B2C_COLOR_CACHE 4        /* reuse the colouring while pairs and masses are unchanged */
#define B2C_COLOR_WARM_START 8   /* warm start by feature key */
#define B2C_COLOR_FIRST_FIT 32   /* Jones-Plassmann with first-fit colours: a pair that wins its
                                     round takes the smallest colour not used around its bodies
                                     (the greedy colouring in priority order: at least the largest
                                     pair count D of one body, at most 2D - 1 colours, and <= 64)
                                     instead of the round number.  Not in the reference; the box
                                     engine's default, as it needs fewer colour phases. */
#define B2C_COLOR_ROW_FORM 64     /* pair solve in row form: the angular response IA (r x d) of every
                                     contact direction, the reciprocal effective masses and the
                                     position bias computed once per substep, so an impulse j along
                                     d changes w by j k.  Not in the reference (whose chunks recompute
                                     IA (r x (j d)) and divide by the effective mass every sweep);
                                     needs B2C_COLOR_FIXED_FRAME.  The box engine's default. */
#define B2C_COLOR_PER_CONTACT 16 /* no manifold reduction; every contact is its own chunk and is
                                    coloured on the contact graph (the plain coloured engine) */
#define B2C_COLOR_REDUCED_CONTACTS 128 /* the manifold reduction, then every kept contact is its own
                                    chunk, coloured with the reduced set's priority (COL:776-787:
                                    its slot inside its run of one body pair, then the parity of
                                    that run, then its rank; the smaller first) -- the reference's
                                    GraphColoredContactEngine(manifold_reduce=True,
                                    pair_chunks=False).  Needs b2c_pairs.prio_hi and a pair
                                    capacity of one per contact. */

#define B2C_COLOR_ISLANDS 256    /* the island solve (IslandSolveContactEngine,
                                    contact_engine_gpu_island_solve.py:253-291): the pair graph is
                                    partitioned into islands of dynamic bodies on the device
                                    (recomputed on every colour-cache miss); when no island has more
                                    than B2C_ISLAND_MAX_PAIRS pairs, one thread per island runs its
                                    warm start, velocity sweeps and (on another thread) position
                                    sweeps over its pairs in colour order, with no barrier between
                                    colours -- the same bits as the persistent solve, which runs
                                    instead when an island is larger.  Needs b2c_pairs.isl_work. */
#define B2C_ISLAND_MAX_PAIRS 64  /* largest island the island solve takes (the reference's 64) */

#define B2C_SOLVE_SCENES 0x100000 /* b2c_color_params.solve_blocks: the scene schedule */

typedef struct b2c_color_params {
    int32_t vit, pit;        /* velocity / position sweeps */
    int32_t max_points;      /* manifold points kept per pair (<= 8) */
    int32_t flags;           /* B2C_COLOR_* */
    float mu;                /* friction */
    float t2d;               /* cross-slip damping of the chunk sweep (1 = full) */
    int32_t color_cap;       /* error when the pair graph needs more colours (<= max_colors) */
    int32_t solve_blocks;    /* persistent solve shape: 0 = pick from the body count; n > 0 = n CTAs
                                with a grid barrier (1 = one CTA, block barriers); -n = a thread-block
                                cluster of n CTAs with the hardware cluster barrier;
                                B2C_SOLVE_SCENES = one CTA per scene (b2c_pairs' scene schedule) */
    int64_t barrier_timeout_ns; /* grid-barrier wait limit */
    const float *body_mu;    /* (bodies) per-body friction, or NULL for the scalar mu: a body pair's
                                contacts use sqrt(mu_a mu_b), a ground pair mu_a */
} b2c_color_params;

/* ---- version / errors ---- */
B2C_API int32_t b2c_version(void);
B2C_API const char *b2c_last_error(void);
/* kernel nodes in a captured cudaGraph_t (child graphs included); -1 on error.  Used to report
 * how many of this library's kernels one replayed step launches. */
B2C_API int32_t b2c_graph_kernel_nodes(void *graph);
/* floats of b2c_pairs.rec for `pair_capacity` pairs of up to `kslots` contacts each */
B2C_API int64_t b2c_pair_record_floats(int32_t pair_capacity, int32_t kslots);
/* B2C_BARRIER_WORDS, the uint32 words a grid-barrier buffer needs */
B2C_API int32_t b2c_barrier_words(void);
/* ints of scratch that b2c_exclusive_scan needs for n elements */
B2C_API int32_t b2c_scan_scratch_ints(int32_t n);
/* exclusive prefix sum of n int32 (device pointers); out may alias nothing */
B2C_API int32_t b2c_exclusive_scan(const int32_t *in, int32_t *out, int32_t n, int32_t *scratch, b2c_stream s);
/* Exclusive scan that allocates nothing and takes no scratch argument: for callers that cannot
 * allocate device memory or own a scratch buffer -- a foreign-language binding that holds only
 * the two arrays it passes, or a host loop that must not allocate once it runs.  No counterpart
 * in the reference (its scans are Warp's array_scan on Warp-allocated arrays).  The scratch is
 * one library-owned device array per device for at most b2c_scan_noalloc_max_n() = 2^24
 * elements; larger n returns B2C_EARG with a message.  Calls share that array: two calls that
 * overlap in time (concurrent streams or host threads) race, so order them on one stream.  The
 * first call on a device looks up the array's address; make it before any stream capture begins
 * on that device.  A call with n = 0 does only that, and accepts null in and out.  The address
 * is cached per device and per CUDA context: after cudaDeviceReset the next call looks it up
 * again, so make that call before a capture too. */
B2C_API int32_t b2c_exclusive_scan_noalloc(const int32_t *in, int32_t *out, int32_t n, b2c_stream s);
B2C_API int32_t b2c_scan_noalloc_max_n(void);

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

/* ---- coloured Gauss-Seidel chain (contact_engine_gpu_colored.py, ColorCache descendants) ---- */
/* k_gen_fid (COL:102-122) + the feature-key radix sort and gather (COL:1057-1061), done as one
 * deterministic pass: per-bead counts, a scan, then each bead writes its ground contact and its
 * neighbours in ascending bead order at its offset.  The output is in feature-key order. */
B2C_API int32_t b2c_bead_contacts_sorted(const b2c_beads *beads, const b2c_grid *g, b2c_contacts *c,
                                         b2c_manifold *m, b2c_header *hdr, b2c_stream s);
/* Pair-key grouping (COL:1062-1064), warm start (k_warm COL:601-626), E-optimal selection
 * (k_select COL:651-728), compaction (k_compact COL:730-751) and the kept-contact pair build
 * (COL:1158-1176).  `kept` receives the kept contacts in feature order with their impulses. */
B2C_API int32_t b2c_manifold_reduce(const b2c_bodies *b, const b2c_beads *beads, const b2c_contacts *c,
                                    b2c_manifold *m, b2c_contacts *kept, int64_t *kept_keys, b2c_pairs *pr,
                                    const b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p, b2c_stream s);
/* Jones-Plassmann colouring of the pair graph (COL:1178-1208) behind the colour cache
 * (contact_engine_gpu_color_cache.py:37-54), entirely on the device. */
B2C_API int32_t b2c_color_pairs(const b2c_bodies *b, b2c_pairs *pr, b2c_header *hdr, const b2c_color_params *p,
                                b2c_stream s);
/* The pair-chunk solve of one substep as one persistent kernel: applied warm start per colour
 * (applied_warm.py:68-75), vit velocity sweeps (fixed frame, fixed_frame.py:7-77, or slip basis,
 * COL:413-490) and pit position sweeps (COL:510-554) over the colours, a bounded grid barrier
 * between colours. */
B2C_API int32_t b2c_color_solve(const b2c_bodies *b, b2c_contacts *kept, b2c_pairs *pr, b2c_header *hdr,
                                const b2c_color_params *p, float dt, b2c_stream s);
/* ints of the island workspace (b2c_pairs.isl_work, b2c_island_partition's work) */
B2C_API int64_t b2c_island_work_ints(int32_t n_bodies, int32_t pair_capacity);
/* partition_pairs (contact_engine_gpu_island_solve.py:7-34) on the device: the pairs
 * (pbi[p], pbj[p]) of bodies with inverse masses inv_mass, taken in the order `order` (a
 * permutation of the n_pairs pairs, or NULL for 0..n_pairs-1), grouped into islands.  Two dynamic
 * bodies (inverse mass > 0) of one pair are in one island; static bodies and the ground (pbj < 0)
 * join nothing.  Writes, in the reference's output order (islands by their smallest body, a pair
 * without a dynamic body keyed bodies + p; each island's pairs in `order`):
 *   packed (n_pairs) the pair indices island by island, starts / counts (n_pairs room) each
 *   island's offset into packed and its pair count, info[0] the number of islands, info[1] the
 *   most pairs of one island (info: 4 device ints).
 * work: b2c_island_work_ints(n_bodies, n_pairs) device ints.  The arguments are not validated
 * on the device (the reference raises ValueError for bad shapes, negative or non-finite masses,
 * endpoints out of range and a non-permutation order; the Python wrapper checks them). */
B2C_API int32_t b2c_island_partition(const int32_t *pbi, const int32_t *pbj, const float *inv_mass,
                                     const int32_t *order, int32_t n_pairs, int32_t n_bodies, int32_t *work,
                                     int32_t *packed, int32_t *starts, int32_t *counts, int32_t *info,
                                     b2c_stream s);
/* _store_warm_device (COL:1089-1093). */
B2C_API int32_t b2c_warm_store(const b2c_contacts *kept, const int64_t *kept_keys, b2c_warm *warm,
                               const b2c_header *hdr, b2c_stream s);
/* One whole ColorCache / pair-chunk substep: predict, beads, grid, sorted contacts, manifold,
 * pairs, colouring (cached), solve, warm store, integrate.  vgrav receives the velocity after
 * gravity (the deferred-force reference point, deferred_force.py:33). */
B2C_API int32_t b2c_color_substep(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, b2c_contacts *c,
                                  b2c_manifold *m, b2c_contacts *kept, int64_t *kept_keys, b2c_pairs *pr,
                                  b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p, float dt,
                                  float *vgrav, b2c_stream s);

/* ---- box engine: body-AABB broadphase + box/plane and box/box narrowphase ---- */
/* Candidate pairs from a uniform hash grid over the body centres: per body its ground
 * candidate (when its AABB reaches z < margin) and every later body whose AABB overlaps, in
 * ascending order (the reference tests all pairs, BoxWorld.contacts, ncp_gpu.py:1273-1280). */
B2C_API int32_t b2c_box_candidates(const b2c_bodies *b, b2c_boxes *bx, b2c_header *hdr, b2c_stream s);
/* float64 SAT per candidate (box_plane_contacts / box_box_contacts, ncp_gpu.py:1148-1227), then
 * compaction into kept contacts (pair order, feature order inside a pair, point on both bodies,
 * depth = -gap) with warm-started impulses, and the pair arrays of the coloured solve. */
B2C_API int32_t b2c_box_contacts(const b2c_bodies *b, b2c_boxes *bx, b2c_contacts *kept, int64_t *kept_keys,
                                 b2c_pairs *pr, const b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p,
                                 b2c_stream s);
/* One box-engine substep: predict, candidates, narrowphase, colouring (cached), the persistent
 * chunk solve, warm store, integrate. */
B2C_API int32_t b2c_box_substep(const b2c_bodies *b, b2c_boxes *bx, b2c_contacts *kept, int64_t *kept_keys,
                                b2c_pairs *pr, b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p,
                                float dt, float *vgrav, b2c_stream s);
/* One box pair / one box and the ground through the device narrowphase (for parity checks):
 * inputs (n,4) half, x, q for a and b; per pair up to 8 points (8,4 = point|gap), a normal
 * (4), 8 feature ids and a count.  b_half == NULL means box a against the ground. */
B2C_API int32_t b2c_box_narrowphase_test(int32_t n, const float *a_half, const float *a_x, const float *a_q,
                                         const float *b_half, const float *b_x, const float *b_q, float margin,
                                         double *pts, double *nrm, int32_t *fid, int32_t *count, b2c_stream s);

/* ---------------------------------------------------------------------------------------------
 * Exact-cone NCP solve (src/motion_engine/ncp/ncp_gpu.py:361-1063, NCPSolverGPU): per-contact
 * 3x6 Jacobian blocks, per-body 6x6 inverse mass, coloured projected Gauss-Seidel on the
 * Coulomb cone with the de Saxce correction, int64 fixed-point per-body accumulation of
 * Minv J^T lambda, optional soft step.  Reals are float32 or float64 (dtype = 4 or 8 bytes).
 * ------------------------------------------------------------------------------------------- */
/* The scene (BlockScene, ncp_gpu.py:193-260), device pointers. */
typedef struct b2c_ncp_scene {
    int32_t n_c, n_b;
    int32_t dtype;             /* bytes of a real: 4 or 8 */
    const void *Ja, *Jb;       /* (n_c,3,6) blocks of body A and B (B carries the minus sign) */
    const void *Minv;          /* (n_b,6,6) */
    const void *v_free;        /* (n_b,6) */
    const void *mu;            /* (n_c) */
    const void *bias;          /* (n_c,3) added to u */
    const void *sep;           /* (n_c) separation, read by the soft step only; may be NULL */
    const int32_t *pa, *pb;    /* (n_c) bodies, -1 = static */
    const int32_t *feature;    /* (n_c) stable feature id (< 2^20), unique per (pa, pb) */
} b2c_ncp_scene;

/* Solver state, device pointers sized by the capacities (NCPSolverGPU.__init__, :799-846). */
typedef struct b2c_ncp_state {
    int32_t max_contacts, n_bodies, max_colors;
    void *rho;                 /* (max_contacts) step 1/lambda_max(W_cc) */
    void *lam;                 /* (max_contacts,3) impulses (n, t1, t2); the warm start on entry */
    void *v;                   /* (n_bodies,6) velocity */
    int64_t *acc;              /* (n_bodies*6) sum_c round(1e10 Minv J_c^T lambda_c) */
    void *res;                 /* (max_contacts) per-contact natural-map residual */
    void *u;                   /* (max_contacts,3) contact velocity of the last residual */
    int32_t *col, *order;      /* (max_contacts) colour of each contact; contacts grouped by colour */
    int32_t *cstart, *ccount;  /* (max_colors) */
    uint64_t *claim;           /* (n_bodies) colouring claims */
    int32_t *dyn;              /* (n_bodies) 1 = dynamic (Minv != 0) */
    int32_t *cache_pa, *cache_pb, *cache_feat; /* (max_contacts) inputs of the cached colouring */
    void *cache_minv;          /* (n_bodies,4) Minv[0][0], [1][1], [2][2] and the dynamic flag */
    int32_t *stats;            /* (8) n_colors, cache_valid, cached_C, cache_hit, hits, misses,
                                  rounds, error bits */
    uint64_t *res_max;         /* (1) bits of max_c residual_c (non-negative reals) */
    uint32_t *barrier;         /* (B2C_BARRIER_WORDS) grid barrier of the persistent sweep */
} b2c_ncp_state;

/* Per-call parameters: de Saxce correction, soft step (SoftStep.params: bias_rate, mass_scale,
 * impulse_scale, inv_h, contact_speed) and its pass flag, colour cache, launch form. */
typedef struct b2c_ncp_params {
    int32_t desaxce, soft, use_bias, color_cache;
    int32_t solve_blocks;      /* 0 auto (one CTA up to 16 384 contacts, else a grid of every
                                  co-resident CTA), 1 one CTA, -n a cluster of n CTAs, n > 1 a
                                  cooperative grid of n CTAs (at most the co-resident count) */
    int32_t pad;
    double softp[5];
    int64_t barrier_timeout_ns; /* grid-barrier wait limit (<= 0: 1 s) */
} b2c_ncp_params;

/* rho (k_rho), dynamic flags, acc = 0 or the warm start scattered (k_scatter), v = v_free +
 * acc / 1e10 (k_apply).  warm != 0: state->lam holds the warm start. */
B2C_API int32_t b2c_ncp_setup(const b2c_ncp_scene *sc, b2c_ncp_state *st, int32_t warm, b2c_stream s);
/* Colouring behind the colour cache (NCPSolverGPU._color_cached / _color, :876-963). */
B2C_API int32_t b2c_ncp_color(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                              b2c_stream s);
/* iters sweeps over the colours in one persistent launch (k_sweep + k_apply_c per colour). */
B2C_API int32_t b2c_ncp_sweeps(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                               int32_t iters, b2c_stream s);
/* Natural-map residual per contact, its maximum and the contact velocity u (k_resid). */
B2C_API int32_t b2c_ncp_residual(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                 b2c_stream s);
/* The adjoint of the sweeps at their final iterate (float64 scenes): the implicit-function
 * derivative of lambda* with respect to the free velocity, the bias and the friction, applied to
 * lam_bar (n_c,3, consumed), as `iters` reverse sweeps at lambda* (the Neumann series of
 * (I - dPhi/dlambda)^-T truncated at `iters` terms; dPhi the sweep, NG:485-568).  Needs the
 * colouring of the last b2c_ncp_color and state->u of a b2c_ncp_residual at lambda*.  Adds to
 * vfree_bar (n_b,6), bias_bar (n_c,3) and mu_bar (n_c); v_bar (n_b,6) is scratch.  No counterpart
 * in the reference's NCPSolverGPU; its CPU sensitivity (ncp_ref.py:907-959) is the converged
 * limit on a fixed branch.  The Jacobian blocks and Minv are held (no adjoint of them). */
B2C_API int32_t b2c_ncp_adjoint(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                int32_t iters, double *lam_bar, double *v_bar, double *vfree_bar, double *bias_bar,
                                double *mu_bar, b2c_stream s);
/* b2c_ncp_sweeps (float64 scenes) that also records what every contact update of every sweep
 * started from, b2c_ncp_trace_words() doubles per update: trace[W (it n_c + c) + 0..2] = the
 * contact's impulse, [3..8] and [9..14] = the velocities (n_b,6 rows) of its bodies pa, pb (zero
 * where there is none); the rest of each record is b2c_ncp_adjoint_unrolled's.  trace_len >= W
 * iters n_c.  The impulses and velocities it leaves are bitwise those of b2c_ncp_sweeps. */
B2C_API int32_t b2c_ncp_trace_words(void);
B2C_API int32_t b2c_ncp_sweeps_record(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                      int32_t iters, double *trace, int64_t trace_len, b2c_stream s);
/* The exact reverse of setup (warm or cold) and the `iters` sweeps recorded by
 * b2c_ncp_sweeps_record (same scene, same colouring, hard contacts): lam_bar (n_c,3) holds the
 * adjoint of the final impulses on entry and that of the starting impulses (the warm start) on
 * return; adds to vfree_bar (n_b,6), bias_bar (n_c,3), mu_bar (n_c), and to the adjoints of the
 * Jacobian blocks Ja_bar, Jb_bar (n_c,3,6) and of Minv_bar (n_b,6,6) -- through the contact
 * velocities, the velocity changes and the step sizes rho_c = 1 / lambda_max(W_c) (where that
 * eigenvalue is simple).  v_bar (n_b,6) is scratch; state->res is overwritten.  The derivative of
 * what the sweeps computed, converged or not: where the converged impulses are not unique
 * (redundant contacts) the one the sweeps reach depends on where they started, which the implicit
 * form above cannot see.  No counterpart in the reference. */
B2C_API int32_t b2c_ncp_adjoint_unrolled(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                         int32_t iters, double *trace, int64_t trace_len, double *lam_bar,
                                         double *v_bar, double *vfree_bar, double *bias_bar, double *mu_bar,
                                         double *Ja_bar, double *Jb_bar, double *Minv_bar, b2c_stream s);

/* ---------------------------------------------------------------------------------------------
 * The exact-cone box world: the reference's BoxWorld substep (src/motion_engine/ncp/ncp_gpu.py:
 * 1237-1413) on the device, in float64, for one scene or many independent ones (the scene ids of
 * b2c_boxes): SAT contacts -> build_scene -> the NCP above -> integration.  A substep is
 *   b2c_world_contacts; (read *count); b2c_world_scene; [b2c_world_warm]; b2c_ncp_setup /
 *   _color / _sweeps; [b2c_world_store]; b2c_world_integrate(state->v)
 * with the NCP scene's pa / pb the world's contact arrays.  Kinematic bodies (kin = 1) have zero
 * inverse mass and move with their prescribed velocity vkin.
 * ------------------------------------------------------------------------------------------- */
typedef struct b2c_world {
    int32_t n;                 /* bodies */
    int32_t max_contacts;
    double *x, *q, *v, *w;     /* (n,3), (n,4) (x, y, z, w), (n,3), (n,3): the state */
    const double *half;        /* (n,3) half extents */
    const double *mass;        /* (n) */
    const double *Ib;          /* (n,3) principal moments m/12 (h_y^2 + h_z^2, ...) (Box.Ib, :1105-1109) */
    const int32_t *kin;        /* (n) 1: kinematic */
    const double *vkin;        /* (n,6) velocity of the kinematic bodies */
    const double *body_mu;     /* (n) friction per body (pair: sqrt(mu_a mu_b), ground: mu_a), or NULL */
    double mu;                 /* friction of every contact when body_mu is NULL */
    float *xc32;               /* (n,4) float32 centres for the broadphase (b2c_boxes.half float32 too) */
    double *x4, *half4;        /* (n,4) scratch: padded centres and half extents */
    double *slot_p;            /* (candidate cap x 8, 4) contact point | gap */
    double *slot_n;            /* (candidate cap, 4) normal of the candidate's contacts */
    int32_t *slot_f;           /* (candidate cap x 8) feature id */
    int32_t *pa, *pb, *fid;    /* (max_contacts) bodies (pb -1: ground), feature id (< 256) */
    int64_t *key;              /* (max_contacts) (pa (n + 1) + pb + 1) 256 + fid, ascending */
    double *p, *nrm, *gap;     /* (max_contacts,3), (max_contacts,3) from pb to pa, (max_contacts) */
    int32_t *attach;           /* (max_contacts) what the contact moves with: bits 0-1 the point (0 pa,
                                  1 pb, 2 between a corner of each), bits 2-3 the normal (0 fixed,
                                  1 pa, 2 pb) -- read by the adjoint */
    int32_t *count;            /* (1) contacts of the last b2c_world_contacts (may exceed max_contacts) */
    int64_t *warm_keys;        /* (max_contacts) warm store: keys of the last stored substep ... */
    double *warm_lam;          /* (max_contacts,3) ... their impulses */
    int32_t *warm_n;           /* (1) */
} b2c_world;

/* box_plane_contacts / box_box_contacts (:1148-1227) over the broadphase candidates of bx
 * (b2c_box_candidates on the float32 mirror), in float64; contacts compacted in candidate order. */
B2C_API int32_t b2c_world_contacts(b2c_world *wd, b2c_boxes *bx, b2c_header *hdr, b2c_stream s);
/* build_scene (:1291-1330) for the first n_contacts contacts: Ja, Jb (n_c,3,6), bias (n_c,3),
 * mu, feature (n_c); Minv (n,6,6) and v_free (n,6) of every body (gravity on when gravity != 0). */
B2C_API int32_t b2c_world_scene(const b2c_world *wd, int32_t n_contacts, double dt, int32_t gravity, double *Ja,
                                double *Jb, double *Minv, double *vfree, double *bias, double *mu, int32_t *feature,
                                b2c_stream s);
/* lam (n_c,3) <- the warm store's impulse of the same key, else 0 (BoxWorld._warm, :1381-1384). */
B2C_API int32_t b2c_world_warm(const b2c_world *wd, int32_t n_contacts, double *lam, b2c_stream s);
/* The transpose of b2c_world_warm between two substeps: lam_bar (n_c,3) of this substep's contacts
 * += tlam of the entry of the table (tkeys ascending, *tn entries, on the device) with the same
 * key -- the table holding the next substep's contact keys and the adjoint of its warm start. */
B2C_API int32_t b2c_world_warm_adjoint(const b2c_world *wd, int32_t n_contacts, const int64_t *tkeys,
                                       const double *tlam, const int32_t *tn, double *lam_bar, b2c_stream s);
/* warm store <- the contacts' keys and lam (:1393-1394). */
B2C_API int32_t b2c_world_store(b2c_world *wd, int32_t n_contacts, const double *lam, b2c_stream s);
/* v, w <- v6 (n,6); x += v dt; q <- normalize(q + 0.5 (w, 0) q dt) (:1399-1406). */
B2C_API int32_t b2c_world_integrate(b2c_world *wd, const double *v6, double dt, b2c_stream s);
/* The adjoint of one substep, in two halves around b2c_ncp_adjoint_unrolled.  The world holds the
 * state before the substep, the NCP scene and state its recorded solve (V6 = the solved
 * velocities).  begin: from the adjoints of the substep's result (xb_out (n,3), qb_out (n,4),
 * vb_out, wb_out (n,3)) the integration's reverse into xb_in, qb_in (partial), Vb = vfree_bar
 * (n,6) and lam_b (n_c,3) = J Minv Vb.  end (lam, V6: the solved impulses and velocities; Vb of
 * begin; Ja_b, Jb_b (n_c,3,6) and Minv_b (n,6,6) of b2c_ncp_adjoint_unrolled): the bias through
 * the gaps, the Jacobian blocks through the lever arms, the contact point and frame (the normal
 * turning with its body, attach), the world inertias, and mu_c = sqrt(mu_a mu_b) onto the bodies
 * -- summed per body with float64 atomics (acc: n x 8 doubles, zero on entry and on return; the
 * order of the additions can move the last bits) -- giving xb, qb
 * (completed), vb, wb of the state before the substep, and mub_body (n, accumulated; may be
 * NULL).  No counterpart in the reference. */
B2C_API int32_t b2c_world_adj_begin(const b2c_world *wd, const b2c_ncp_scene *sc, const double *V6, double h,
                                    const double *xb_out, const double *qb_out, const double *vb_out,
                                    const double *wb_out, double *xb_in, double *qb_in, double *Vb, double *vfree_b,
                                    double *lam_b, b2c_stream s);
B2C_API int32_t b2c_world_adj_end(const b2c_world *wd, const b2c_ncp_scene *sc, const double *lam, const double *V6,
                                  const double *Vb, double h, const double *bias_b, const double *mu_b,
                                  const double *vfree_b, const double *Ja_b, const double *Jb_b, const double *Minv_b,
                                  double *acc, double *xb, double *qb, double *vb, double *wb, double *mub_body,
                                  b2c_stream s);

/* ---------------------------------------------------------------------------------------------
 * Batched exact-cone NCP in Delassus form and its implicit adjoint (the reference's batched
 * adjoint BatchProxADMMGPU, src/motion_engine/ncp/ncp_batch_gpu.py:918-1313, and its CPU
 * implicit-function sensitivity, src/motion_engine/ncp/ncp_ref.py:786-959).  float64.  Every
 * environment e has n_c[e] <= 16 contacts; arrays are padded to n_max = 3 x (max n_c) rows.
 * ------------------------------------------------------------------------------------------- */
typedef struct b2c_bncp {
    int32_t n_env;
    int32_t n_max;          /* rows per environment, a multiple of 3, <= b2c_bncp_max_rows() */
    const int32_t *nc;      /* (n_env) contacts of each environment */
    const double *G;        /* (n_env, n_max, n_max) Delassus J Minv J^T, row-major */
    const double *b;        /* (n_env, n_max) free contact velocity J v_free + bias */
    const double *mu;       /* (n_env, n_max/3) friction */
    double *lam;            /* (n_env, n_max) warm start in, solution out (n, t1, t2 per contact) */
    double *res;            /* (n_env) natural residual of the returned lambda */
    int32_t *iters;         /* (n_env) sweeps run (the convergence mask: < max_iters = converged) */
    int32_t *labels;        /* (n_env, n_max/3) 0 open, 1 stick, 2 slip (written by the adjoint) */
    int32_t *status;        /* (n_env) 1 = singular branch, 2 = branch boundary (responses NaN) */
} b2c_bncp;

B2C_API int32_t b2c_bncp_max_rows(void);
/* Projected Gauss-Seidel per environment until the natural residual < tol (checked every
 * `check` sweeps) or max_iters (ncp_batch_gpu.py's convergence mask; ncp_gpu.py:485-568 sweep). */
B2C_API int32_t b2c_bncp_solve(const b2c_bncp *p, int32_t max_iters, double tol, int32_t check, b2c_stream s);
/* Full fixed-branch responses dlam/dmu (n_env, n_max, n_max/3) and dlam/db (n_env, n_max, n_max)
 * at p->lam (ncp_ref.sensitivity, :907-959); NaN where the branch is singular or on a boundary. */
B2C_API int32_t b2c_bncp_sensitivity(const b2c_bncp *p, double *dlam_dmu, double *dlam_db, b2c_stream s);
/* Vector-Jacobian product at p->lam: gb = (dlam/db)^T glam, gmu = (dlam/dmu)^T glam (the
 * backward of the batched adjoint, ncp_batch_gpu.py:1172-1186). */
B2C_API int32_t b2c_bncp_vjp(const b2c_bncp *p, const double *glam, double *gb, double *gmu, b2c_stream s);

/* ---------------------------------------------------------------------------------------------
 * Batched proximal ADMM with its adjoint: the reference's BatchProxADMMGPU
 * (src/motion_engine/ncp/ncp_batch_gpu.py:918-1313).  n_env independent problems of nc point
 * contacts on nv generalised velocities each (J: 3 nc x nv rows n, t1, t2 per contact), solved
 * matrix-free (G x = J (M^-1 J^T x), with M^-1 J^T x summed in int64 at a per-problem
 * power-of-two scale, NB:326-388) by ADMM with a block-Jacobi preconditioned CG x-step, the
 * exact cone projection and a per-problem convergence mask; then the fixed-branch adjoint by
 * grad_affine (NB:1172-1186).  One warp per problem runs the whole solve in one launch.
 * ------------------------------------------------------------------------------------------- */
#define B2C_ADMM_MAX_CONTACTS 8
#define B2C_ADMM_MAX_DOFS 32
#define B2C_ADMM_FORWARD 1      /* set-up and n_iter ADMM iterations from zero (NB:1190-1195) */
#define B2C_ADMM_GRADIENT 2     /* then d/dtau_jdir and d/dmu at the first slip contact (NB:1197-1206) */
#define B2C_ADMM_GRAD_GIVEN 4   /* instead of the forward: grad_affine at the given lam and u for the
                                   b-direction dbv_in (the reference's own adjoint test,
                                   tests/test_ncp_batch_adjoint.py:55-76) */
#define B2C_ADMM_RHO_SQRT 0     /* rho = sqrt(lambda_min+ lambda_max) of G (k_rho NB:261-288) */
#define B2C_ADMM_RHO_LMIN 1
#define B2C_ADMM_RHO_LMAX 2
#define B2C_ADMM_RHO_REGIME 3   /* lambda_max when the bilateral solution leaves a cone, else lambda_min+ */
#define B2C_ADMM_RHO_GIVEN 4    /* b2c_admm.rho as given */

typedef struct b2c_admm {
    int32_t n_env, nc, nv;
    const double *J;        /* (n_env, 3 nc, nv) row-major */
    const double *Minv;     /* (n_env, nv, nv) */
    const double *v_free;   /* (n_env, nv); b = J v_free */
    const double *mu;       /* (n_env, nc) */
    double *lam;            /* (n_env, nc, 3) out (FORWARD) or in (GRAD_GIVEN) */
    double *u;              /* (n_env, nc, 3) contact velocity of the last refresh; out or in likewise */
    double *v_plus;         /* (n_env, nv) v_free + M^-1 J^T lam (FORWARD) */
    double *res;            /* (n_env) natural residual of the last refresh, NaN when none ran, or NULL */
    int32_t *mask;          /* (n_env) 1 = still iterating (not below tol), or NULL */
    double *rho;            /* (n_env) the ADMM penalty used (out), or in with B2C_ADMM_RHO_GIVEN; or NULL */
    int32_t *nslip;         /* (n_env) slip contacts of the active set (GRADIENT / GRAD_GIVEN) */
    int32_t *labels;        /* (n_env, nc) 0 open, 1 stick, 2 slip */
    double *dlam_tau;       /* (n_env, nc, 3) dlam for db = dt J M^-1 e_jdir (or for dbv_in) */
    double *dv_tau;         /* (n_env, nv) dv+ for the same direction */
    double *dlam_mu;        /* (n_env, nc, 3) dlam / dmu at each problem's first slip contact */
    const double *dbv_in;   /* (n_env, nc, 3) the b-direction of B2C_ADMM_GRAD_GIVEN, else NULL */
    const double *b_in;     /* (n_env, nc, 3) the free contact velocity b itself, or NULL for J v_free */
} b2c_admm;

typedef struct b2c_admm_params {
    int32_t flags;          /* B2C_ADMM_FORWARD [| B2C_ADMM_GRADIENT] or B2C_ADMM_GRAD_GIVEN */
    int32_t n_iter, cg_iters, refresh_every;
    double tol;             /* a problem freezes once its residual at a refresh is below tol */
    int32_t chunk;          /* > 0: the refresh count restarts every `chunk` iterations (the reference's
                               chunked forward, NB:1112-1143); 0: one block (its step-and-gradient graph) */
    int32_t desax;          /* natural residual with the de Saxce term */
    int32_t rho_mode;       /* B2C_ADMM_RHO_* */
    int32_t jacobi_sweeps;  /* cyclic Jacobi sweeps of G's spectrum (the reference's 10) */
    double alpha_eta;       /* eta = alpha |G_cc| (the reference's default 0) */
    double dt;              /* db = dt J M^-1 e_jdir */
    int32_t jdir;           /* generalised coordinate of the tau direction */
    int32_t n_calls;        /* applications of the sigma map (n_slip max + 2; <= 0: nc + 2) */
    int32_t grad_cg;        /* CG iterations of each application */
    int32_t do_mu;          /* also the mu direction */
} b2c_admm_params;

/* dynamic shared memory of one problem (-1 when nc or nv is out of range) */
B2C_API int64_t b2c_admm_smem_bytes(int32_t nc, int32_t nv);
B2C_API int32_t b2c_admm_solve(const b2c_admm *a, const b2c_admm_params *p, b2c_stream s);

/* ---------------------------------------------------------------------------------------------
 * Engine handle: the ContactEngine protocol (src/motion_engine/contact_engine.py:48-55) as C
 * calls, for callers without a tensor library.  A handle owns its device memory (one
 * allocation, sized at the first step from the bodies added; adding bodies afterwards rebuilds
 * from the added centres, as the reference's add_body does, contact_engine_gpu.py:205-207) and
 * runs b2c_box_substep, the launch sequence the Python box engine runs, so a handle and the
 * Python engine over the same bodies give the same bits.  Kind: the box engine (solid boxes,
 * float64 SAT contacts, the ColorCache pair solve).
 *
 * Centres, sizes, densities and dt are float64 as in the reference's Python setup: the body
 * arrays are computed in float64 and rounded once to float32 (Box.Ib, ncp_gpu.py:1105-1109).
 * Calls without a stream argument run on the stream of the last b2c_step (the legacy default
 * stream before the first) and return when their work is done.  A handle is used from one host
 * thread at a time.
 * ------------------------------------------------------------------------------------------- */
#define B2C_ENGINE_BOX 1

typedef struct b2c_config {
    int32_t kind;               /* B2C_ENGINE_BOX */
    int32_t device;             /* CUDA device ordinal */
    int32_t vit, pit;           /* velocity / position sweeps per substep */
    double mu;                  /* friction of bodies without their own (b2c_set_body_mu) */
    double dims[3];             /* box edges of bodies added without their own */
    double margin;              /* contact margin (the reference's 2e-3) */
    int32_t flags;              /* B2C_COLOR_* (not B2C_COLOR_PER_CONTACT or B2C_COLOR_ISLANDS) */
    int32_t color_cap;          /* colour cap, <= 512 */
    int32_t solve_blocks;       /* launch form of the persistent solve (b2c_color_params) */
    int32_t cand_per_body;      /* candidate pairs reserved per body */
    int64_t barrier_timeout_ns; /* grid-barrier wait limit; <= 0: 1 s */
    int32_t graph;              /* 1: each (dt, substeps) step is captured into a CUDA graph
                                   after its first eager run and replayed afterwards */
} b2c_config;

/* Counters read back by b2c_sync_header (the Python engines' diagnostics attributes). */
typedef struct b2c_step_header {
    b2c_header last;            /* counters of the last substep */
    int32_t color_cache_hits, color_cache_misses;
    int32_t graph_captures;     /* CUDA graphs captured so far */
    int32_t kernels_per_step;   /* kernel nodes of the last captured step graph (0: none yet) */
    int32_t bodies;
    int32_t built;              /* 1 once the device arrays exist */
} b2c_step_header;

/* The box engine's defaults: vit 16, pit 10, mu 0.5, dims 0.3 x 0.3 x 0.2, margin 2e-3, flags
 * fixed frame | apply warm | cache | warm start | first fit | row form, colour cap 512, solve form
 * picked from the body count, 16 candidates per body, 1 s barrier limit, graphs on, device 0. */
B2C_API void b2c_config_init(b2c_config *c);
/* Host-side body arrays of n solid boxes (Box.Ib, ncp_gpu.py:1105-1109): mass = density x the
 * box volume and the diagonal body inertia in float64; xc4 (n,4) centre, invM (n) (0 when
 * kinematic), IbInv12 (n,12) inverse inertia rows (the identity when kinematic), M (n) mass.
 * Host pointers; no device work.  B2C_EARG for a non-positive mass or a non-finite inverse. */
B2C_API int32_t b2c_box_body_setup(int32_t n, const double *center3, const double *dims3, const double *density,
                                   const int32_t *kin, float *xc4, float *invM, float *IbInv12, double *M);
/* Validates the configuration and returns a handle; no device work until the first step. */
B2C_API int32_t b2c_create(const b2c_config *c, void **h);
/* Appends n bodies (add_body / add_box): centres (n,3); densities (n) or NULL (1000); edges
 * (n,3) or NULL (the configured dims); kinematic flags (n) or NULL (none).  Bodies get the
 * configured friction and scene 0. */
B2C_API int32_t b2c_add_bodies(void *h, int32_t n, const double *center3, const double *density, const double *dims3,
                               const int32_t *kin);
/* Per-body friction of bodies [first, first+n): a pair uses sqrt(mu_a mu_b), the ground mu_a. */
B2C_API int32_t b2c_set_body_mu(void *h, int32_t first, int32_t n, const double *mu);
/* Scene of bodies [first, first+n) for a batch of independent scenes (bodies of different
 * scenes never touch; each colours as it would alone). */
B2C_API int32_t b2c_set_body_scene(void *h, int32_t first, int32_t n, const int32_t *scene);
B2C_API int32_t b2c_body_count(const void *h);
/* Live kinematic update (contact_engine_gpu.py:241-249): the body moves to xc3 and gets
 * invM = 0, v = w = 0. */
B2C_API int32_t b2c_set_kinematic(void *h, int32_t i, const double *xc3);
/* Advances dt in `substeps` substeps of dt / substeps, asynchronously on s.  Before launching it
 * reads the previous step's device error bits: if any are set it clears them and returns
 * B2C_ECAPACITY or B2C_ETIMEOUT without stepping (the Python engines raise RuntimeError). */
B2C_API int32_t b2c_step(void *h, double dt, int32_t substeps, b2c_stream s);
/* Waits for the last step and returns its counters. */
B2C_API int32_t b2c_sync_header(void *h, b2c_step_header *out);
/* get_state: xc (n,3), q (n,4) quaternion (x, y, z, w), v (n,3), w (n,3) float32, host or device
 * pointers, any of them NULL to skip. */
B2C_API int32_t b2c_get_state(void *h, float *xc, float *q, float *v, float *w);
/* The whole body state as one (4, n, 4) float32 block (planes xc, q, v, w, rows padded to four
 * floats): one copy on s, asynchronous for pinned host or device memory. */
B2C_API int32_t b2c_get_state_packed(void *h, float *state, b2c_stream s);
B2C_API int32_t b2c_set_state_packed(void *h, const float *state, b2c_stream s);
/* contact_forces: f3 (n,3) float64 host = M (v_after - v_before) / dt of the last substep
 * (deferred_force.py:66-74); kinematic rows 0. */
B2C_API int32_t b2c_contact_forces(void *h, double *f3);
/* Checkpoint: everything a later step reads (body state, masses and kinematic flags, the warm
 * store, the colour cache, the counters), so that a handle over the same bodies and
 * configuration that loads the blob continues bit for bit.  blob == NULL: *size receives the
 * size needed. */
B2C_API int32_t b2c_state_save(void *h, void *blob, size_t *size);
B2C_API int32_t b2c_state_load(void *h, const void *blob, size_t size);
/* Frees the handle and its device memory and sets *h = NULL. */
B2C_API int32_t b2c_destroy(void **h);

#ifdef __cplusplus
}
#endif
#endif /* B2C_H */
