/*
 * meep_b200.h -- C ABI of the B200 (sm_100a) FDTD time-stepping hot path.
 *
 * Plain C: device pointers, sizes and POD descriptors; no torch types. Every
 * entry point returns an mtb status code; mtb_last_error() gives the text of
 * the last failure on the calling thread. Nothing here throws.
 *
 * Each entry point replaces one seam of the reference (meep_torch):
 *
 *   mtb_yee2d_plan_create / mtb_yee2d_run
 *       replace the per-step loop core/run.py:10-40 (_run_chunk) driving
 *       core/stepper_tm.py:234 (step_tm) or core/stepper_te.py:178 (step_te)
 *       together with core/sources.py:90 (soft-source injection) and the
 *       sum-folded monitors of core/monitors.py:24-155; reached through
 *       run_tm / run_te (core/run.py:125-126) and fields.step_n
 *       (mp/cpp/core.py:802). A plan is a batch of independent structures.
 *   mtb_yee3d_plan_create / mtb_yee3d_run
 *       replace the loop core/monitors_3d.py:192-210 (run_3d over
 *       core/stepper_3d.py:303 step_3d, CPML path :363-445, source :448-482)
 *       and core/stepper_3d_lean.py:307 (run_3d_lean), with FluxMonitor3D /
 *       DFTFieldsMonitor3D (core/monitors_3d.py:70-189) accumulation.
 *   mtb_pack / mtb_unpack
 *       move the reference's per-component tensors (TMState / TEState /
 *       State3D, core/stepper_tm.py:12, core/stepper_te.py:11,
 *       core/stepper_3d.py:38) into and out of the padded box layout the
 *       kernels use.
 *
 * Ownership: the caller allocates every field, coefficient, source list and
 * accumulator array (device memory) and keeps it alive while a plan uses it.
 * A plan owns only its scratch (sample ring, phase/amplitude tables, work
 * list), allocated at creation and released by the matching destroy call.
 * Threading: a plan is not re-entrant; use one plan per stream.
 */
#ifndef MEEP_B200_H
#define MEEP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (the Python layer maps them to ValueError /
 * NotImplementedError / RuntimeError like core/coeffs.py:81, :179) */
#define MTB_OK 0
#define MTB_INVALID_ARG 1
#define MTB_UNSUPPORTED 2
#define MTB_DEVICE_TIMEOUT 3
#define MTB_CUDA_ERROR 4

#define MTB_ABI_VERSION 1

/* polarisations */
#define MTB_TM 0
#define MTB_TE 1

/* 2D component ids: 0 = the integer-step field (TM Ez, TE Hz),
 * 1 = the x component (TM Hx, TE Ex), 2 = the y component (TM Hy, TE Ey).
 * Sampling an E component samples E = D / eps, computed in the kernel. */
#define MTB_C2_MAIN 0
#define MTB_C2_X 1
#define MTB_C2_Y 2

/* 3D component ids */
#define MTB_EX 0
#define MTB_EY 1
#define MTB_EZ 2
#define MTB_HX 3
#define MTB_HY 4
#define MTB_HZ 5

/* A soft current as a list of cells sorted by row (CSR over the rows of
 * the target component's box array). The cell (row r, col c) receives
 *     F[r, c] -= amp_tbl[t, amp_col] * w
 * where amp_tbl[t, col] = float32(coef[t][col]) of the run call's FP64
 * coefficient table (dt * amplitude(t) for the reference, rounded once, as
 * core/stepper_tm.py:197-200 computes dt * amp * mask). */
typedef struct mtb_cells {
    const int32_t *row_ptr; /* rows+1 entries, device; NULL = no cells     */
    const int32_t *col;     /* n entries, device; ascending within a row
                               (plans reject other orders)                 */
    const float *w;         /* n entries, device                           */
    int32_t n;              /* number of cells                             */
    int32_t amp_col;        /* amplitude-table column this list reads      */
    int32_t row_lo, row_hi; /* first / last row holding cells; the plan
                               fills these (caller values are ignored)     */
} mtb_cells;

/* One raw line of field values copied into the sample ring each step:
 * kind 0 = a row segment F[index, lo:hi], kind 1 = a column segment
 * F[lo:hi, index]. Element p of the segment goes to
 * ring[slot * slot_elems + ring_off + p]. */
typedef struct mtb_line_sample {
    int32_t comp;     /* MTB_C2_*                                       */
    int32_t kind;     /* 0 = row, 1 = column                            */
    int32_t index;    /* row (kind 0) or column (kind 1)                */
    int32_t lo, hi;   /* segment bounds along the other axis            */
    int32_t pad_;
    int64_t ring_off;
} mtb_line_sample;

/* One 2D structure (one TMState/TMCoeffs or TEState/TECoeffs pair).
 * Box layout: every 2D array is nx rows x pitch floats, row-major, the
 * component's reference array (e.g. Hx of shape (nx, ny-1)) occupying its
 * top-left corner, every other cell zero. pitch >= ny, pitch % 4 == 0, and
 * every base pointer 16-byte aligned.
 * Evolving arrays come in ping-pong pairs [2]: a step reads buffer `cur`
 * and writes buffer cur^1 (a fused H+E pass recomputes halo cells from the
 * old values of its neighbours, so it cannot update in place). Both buffers
 * of a pair start equal; mtb_yee2d_current() says which one is live. */
typedef struct mtb_yee2d_struct {
    int32_t pol;            /* MTB_TM / MTB_TE                              */
    int32_t nx, ny, pitch;
    int32_t y_pmc;          /* TM: PMC walls in y (core/coeffs.py y_pmc)    */
    int32_t explicit_e;     /* TM: 1 = read old Ez from e_explicit this run's
                               first step (imported Ez != Dz/eps)           */
    float dt, dx;
    float *f_main[2];       /* TM Dz | TE Hz                                */
    float *f_x[2];          /* TM Hx | TE Dx                                */
    float *f_y[2];          /* TM Hy | TE Dy                                */
    const float *inv_eps_a; /* 1/eps: TM 1/eps_inf | TE 1/eps_x (E = D/eps
                               is evaluated as D * (1/eps))                 */
    const float *inv_eps_b; /* TM unused  | TE 1/eps_y                      */
    const float *e_explicit;/* TM: Ez box array when explicit_e             */
    /* CPML memory, box layout at the position of the field it feeds:
     * TM: [0] psi_Ezy (Hx), [1] psi_Ezx (Hy), [2] psi_Hyx (Dz), [3] psi_Hxy (Dz)
     * TE: [0] psi_Hzy (Dx), [1] psi_Hzx (Dy), [2] psi_Eyx (Hz), [3] psi_Exy (Hz) */
    float *psi[4][2];
    /* CPML (b, a) profiles, kappa == 1: half nodes along x (nx-1), half
     * nodes along y (ny-1), integer nodes along x (nx), along y (ny). */
    const float *hx_b, *hx_a, *hy_b, *hy_a, *ex_b, *ex_a, *ey_b, *ey_a;
    mtb_cells src_e;        /* TM -> Dz rows | TE -> Dy rows                */
    mtb_cells src_h1;       /* TM -> Hy rows | TE -> Hz rows                */
    mtb_cells src_h2;       /* TM -> Hx rows | TE unused                    */
    const mtb_line_sample *lines; /* device array of line samples          */
    int32_t n_lines;
    int32_t xband[4];       /* plan-filled (caller values ignored): the hx
                               profile is active on rows r < xband[0] or
                               r >= xband[1], the ex profile on rows
                               r < xband[2] or r >= xband[3]              */
    int32_t yband[4];       /* plan-filled: the hy profile is active on
                               columns j < yband[0] or j >= yband[1], the ey
                               profile on j < yband[2] or j >= yband[3]   */
    int32_t pad_;
    int64_t ring_full[3];   /* full-grid sample of comp c to ring offset, -1 = off */
    /* electric conductivity (core/coeffs.py sigma_d; core/stepper_tm.py:158-163,
     * core/stepper_te.py D update): null = none. Box arrays at the D
     * component's position: D' = d1 D + d2 curl H, and the soft current on D
     * is scaled by d2 instead of dt. TM uses [0] (Dz); TE [0] (Dx), [1] (Dy).
     * Tile kernels only (variant 2); other variants and the adjoint return
     * MTB_UNSUPPORTED. */
    const float *cond_d1[2];
    const float *cond_d2[2];
    /* dispersive poles (ADE Lorentz / Drude; TM core/stepper_tm.py:203-231, TE
     * core/stepper_te.py:136-175): n_poles (<= MTB_MAX_POLES) planes of
     * nx x pitch floats each, plane k at k * nx * pitch, on TM Ez or TE Ex.
     * pol_p[3] rotate: with s = mtb_yee2d_pole_slot(plan) (0 at creation, +1
     * mod 3 per step), buffer s holds P(n), buffer (s+2)%3 P(n-1), and the step
     * writes P(n+1) = c1 P(n) + c2 P(n-1) + c3 E(n) into buffer (s+1)%3 (three
     * buffers, because TE recomputes its neighbours' P(n+1) from their P(n-1));
     * then E(n+1) = (D(n+1) - sum_k P_k(n+1)) / eps. pol_c = c1, c2, c3.
     * TE's Ey poles are the second set (n_poles_y, pol_py, pol_cy). Tile
     * kernels only (variant 2); the other variants and the adjoint return
     * MTB_UNSUPPORTED. */
    int32_t n_poles;
    int32_t n_poles_y;
    float *pol_p[3];
    const float *pol_c[3];
    float *pol_py[3];
    const float *pol_cy[3];
    /* Magnetic conductivity / permeability (core/coeffs.py:161-175, :410-414):
     * H' = h1 H - h2 curl E (TM Hx, TE Hz) or h1 H + h2 curl E (TM Hy), with
     * h1 = (1 - sigma_b dt/2) / (1 + sigma_b dt/2), h2 = dt / (mu (1 + sigma_b dt/2))
     * Yee-averaged onto the H nodes. TM: slot 0 = Hx (h1x, h2x), slot 1 = Hy
     * (h1y, h2y); TE: slot 0 = Hz (hz1, hz2), slot 1 unused. Box layout like
     * the field; NULL = the plain step (h1 = 1, h2 = dt). Tile kernels only
     * (variant 2); the other variants and the adjoint return MTB_UNSUPPORTED. */
    const float *mag_h1[2];
    const float *mag_h2[2];
    /* Symmetry cuts at the low-y / low-x edges (core/coeffs.py:148-285 y_mirror,
     * x_mirror, y_rot2, rot4 and :375-503; core/stepper_tm.py:85-166,
     * core/stepper_te.py:73-111). The cut row / column of the D component is
     * live and the far wall stays PEC. cut_y / cut_x:
     *   0  no cut;
     *   1  TM: the H ghost beyond the cut is zero (even mirror);
     *      TE: the D row on the cut takes dHz/dn = 2 Hz / dx (even mirror;
     *      an odd TE mirror changes only the CPML profiles: pass 0);
     *   2  TM: the on-plane H line beyond the cut is live (odd mirror, Rotate2,
     *      Rotate4), held in f_x0 (nx floats, the Hx row at the y cut) or
     *      f_y0 (ny floats, the Hy column at the x cut) and advanced from the
     *      ghost Ez = cut_ph * Ez(partner): cut_map 0 = the cut cell itself,
     *      1 = reversed along the cut (Rotate2, y cut only), 2 = the transposed
     *      cell of the other cut (Rotate4, square grids).
     * The caller packs the E-side CPML memory and the (b, a) node profiles
     * from the cut row (offset 0). Tile kernels only (variant 2); the other
     * variants and the no-alloc entry return MTB_UNSUPPORTED; the adjoint takes
     * every cut (cut 2 with mtb_adj2d_buffers.g_cut). */
    int32_t cut_y, cut_x;
    int32_t cut_map_y, cut_map_x;
    float cut_ph_y, cut_ph_x;
    int32_t pad2_[2];
    float *f_x0[2];
    float *f_y0[2];
    /* TM instantaneous chi2 / chi3 (core/coeffs.py:155-158; core/stepper_tm.py:222-230):
     * box arrays of chi2, chi3 and eps_inf (all three, or all null = linear). Ez is
     * then the fixed point rhs / (eps + chi2 Ez + chi3 Ez^2) after three sweeps from
     * rhs / eps, rhs = Dz - sum P, wherever the step reads or writes Ez. Tile kernels
     * only (variant 2); other variants, the no-alloc entry and the adjoint return
     * MTB_UNSUPPORTED. */
    const float *chi2, *chi3, *eps_nl;
    const void *pad3_;
    /* TM magnetic Lorentz poles (core/coeffs.py:177-193; core/stepper_tm.py:114-117,
     * :186-196, :209-219): n_mpoles (<= MTB_MAX_POLES) on Hx (slot 0) and Hy (slot 1).
     * B integrates the curl (B' = B -/+ dt curl, CPML as for H), the magnetic sheet
     * sources go into B, M(n+1) = mc1 M(n) + mc2 M(n-1) + mc3 H(n-1/2) and
     * H(n+1/2) = B(n+1/2) - sum_k M_k(n+1). f_b[c][2]: B, ping-pong box arrays like
     * f_x / f_y; mpol[c][3]: stacks of n_mpoles planes rotating like pol_p (buffer s =
     * mtb_yee2d_pole_slot holds M(n), (s+2)%3 M(n-1), (s+1)%3 receives M(n+1));
     * mpc[c][3]: mc1, mc2, mc3 stacks. No magnetic conductivity pairs and no live
     * symmetry-cut lines with them (core/coeffs.py:177-179, :240-244). Tile kernels
     * only (variant 2) and the adjoint (mtb_adj2d_buffers.g_b / g_mpol); other
     * variants and the no-alloc entry return MTB_UNSUPPORTED. */
    int32_t n_mpoles;
    int32_t pad4_[3];
    float *f_b[2][2];
    float *mpol[2][3];
    const float *mpc[2][3];
    /* TE in-plane tensor eps and oriented poles (core/coeffs.py:389-399, :428-456;
     * core/stepper_te.py:136-175): te3 = 1 runs the structure as three passes (D and
     * poles, E, Hz) with E stored in e_x (Ex, nx-1 x ny) and e_y (Ey, nx x ny-1), box
     * layout, one buffer each, holding the state's E between steps. tinv: inv_xx and
     * inv_xy at the Ex nodes, inv_yy and inv_xy at the Ey nodes (null: E = rhs / eps
     * from inv_eps_a / inv_eps_b). c3xy / c3yx: the oriented poles' cross drives of Px
     * by the four-node average of Ey and of Py by that of Ex, stacks like pol_c / pol_cy
     * (null = none). Tile kernels only (variant 2); other variants, the no-alloc entry
     * and the adjoint return MTB_UNSUPPORTED. */
    int32_t te3;
    int32_t pad5_[3];
    const float *tinv[4];
    float *e_x, *e_y;
    const float *c3xy, *c3yx;
    /* TE instantaneous chi2 / chi3 on the three-pass kernels (te3 = 1; core/coeffs.py:
     * 380-387, core/stepper_te.py:160-174): nlx = chi2, chi3, eps at the Ex nodes, nly
     * the same at the Ey nodes (box layout; all null = linear). E starts at rhs / eps and
     * takes three Jacobi sweeps E = rhs / (eps + chi2 E + chi3 (E^2 + avg4(E_other)^2)),
     * through the scratch boxes e_t (Ex, Ey). Not with the tensor eps. */
    const float *nlx[3];
    const float *nly[3];
    float *e_t[2];
} mtb_yee2d_struct;

#define MTB_MAX_POLES 8

/* A DFT phase group: frequencies sharing one table. The plan evaluates
 *   P(t, f, s) = dt * (cos(w (t + s/2) dt), -sin(w (t + s/2) dt)),  s in {1, 2}
 * in FP64 (mode 0) or with the reference's float32 phase arithmetic
 * w = float32(2 pi) * float32(f), float32(w * float32(t)) (mode 1,
 * core/monitors.py:43-46), then rounds to float32. */
typedef struct mtb_phase_group {
    const double *freqs;    /* host pointer, nf entries                     */
    int32_t nf;
    int32_t mode;
    double dt;
} mtb_phase_group;

/* A DFT accumulation region: rows x cols sample channels read from the
 * ring (offset a, optionally averaged 0.5*(a+b) with offset b, as the flux
 * monitors average H across the plane), folded into a caller accumulator:
 *   acc[re_off + f*f_stride + r*acc_pitch + c] += sum_t Re P(t,f) * x
 *   acc[im_off + f*f_stride + r*acc_pitch + c] += sum_t Im P(t,f) * x
 * toff = 1 samples at (t + 1/2) dt, toff = 2 at (t + 1) dt. */
typedef struct mtb_dft_region {
    float *acc;             /* device accumulator base                      */
    int64_t re_off, im_off, f_stride;
    int64_t ring_a, ring_b; /* ring offsets; ring_b = -1: no averaging      */
    int32_t rows, cols;
    int32_t ring_pitch, acc_pitch;
    int32_t group, toff;
} mtb_dft_region;

/* Tuning knobs (0 = library default). */
typedef struct mtb_tuning {
    int32_t rows_per_warp;  /* 2D tiles: rows per warp (>= 4: four, register-
                               blocked; 1-3: one; 0: four when the batch fills
                               the GPU, else one); 2D row march: rows one warp
                               marches through; 3D fused: x planes one block
                               covers; 3D split: x planes per H / E launch pair
                               (0 = all)                                     */
    int32_t ring_slots;     /* steps buffered before one DFT contraction    */
    int32_t graph;          /* 2D: replay whole ring flushes (ring_slots steps
                               + one contraction) as a CUDA graph: 0 default
                               (every whole flush after the plan's first step
                               while per-launch timing is off), -1 off      */
    int32_t variant;        /* 2D: 0 default (3 when every structure is
                               eligible, else 2), 1 row march, 2 one-step
                               tiles, 3 temporally blocked tiles (up to 4
                               steps per launch from TMA-staged 32 x 128
                               tiles; PEC structures without conductivity,
                               poles or magnetic pairs; the plan's first
                               step runs on the one-step tiles);
                               3D: 0 default (3 where it applies, else 2),
                               1 fused x-march (register-staged), 2 split
                               H / E streaming kernels, 3 one-pass x-march
                               (H and E of a plane in one kernel from
                               TMA-staged planes; no damping or poles,
                               zpitch <= 256; half steps and x slabs move
                               a default plan to 2)                         */
    int32_t geometry;       /* 3D one-pass kernel work split: 0 default and 1
                               tile-major shares of equal cost, 2 lockstep
                               (every tile cut at the same x planes, tile
                               heights balanced by cost: fewer DRAM bytes,
                               more issue slots)                            */
} mtb_tuning;

typedef struct mtb_yee2d_plan mtb_yee2d_plan;

/* Create a plan for n_structs structures. `structs`, `regions`, `groups`
 * are host arrays copied by the call. ring_slot_elems is the number of
 * floats one step of samples occupies (max ring offset + extent). */
int mtb_yee2d_plan_create(const mtb_yee2d_struct *structs, int32_t n_structs,
                          const mtb_dft_region *regions, int32_t n_regions,
                          const mtb_phase_group *groups, int32_t n_groups,
                          int64_t ring_slot_elems, int32_t n_amp_cols,
                          const mtb_tuning *tuning, mtb_yee2d_plan **out);

/* Advance every structure k steps, t0 .. t0+k-1 (t is the reference's
 * t_idx). coef_e / coef_h: host arrays [k][n_amp_cols] of per-step mask
 * coefficients in FP64 -- for the reference that is dt * source.amplitude(t)
 * (resp. dt * h_amplitude(t)); the plan rounds them to float32. NULL if
 * unused. All monitor contributions of the k steps are folded into the
 * accumulators before the call's work completes on `stream`. */
int mtb_yee2d_run(mtb_yee2d_plan *plan, int64_t t0, int32_t k,
                  const double *coef_e, const double *coef_h, void *stream);

/* Which buffer of every ping-pong pair holds the current state (0 or 1). */
int32_t mtb_yee2d_current(const mtb_yee2d_plan *plan);
/* The pole buffer holding P(n) now (mtb_yee2d_struct.pol_p / pol_py). */
int32_t mtb_yee2d_pole_slot(const mtb_yee2d_plan *plan);

/* Run ONE 2D structure k steps without allocating anything (no counterpart
 * in the reference). For callers that must not call cudaMalloc / cudaFree:
 * a host that gives this library a fixed device-memory budget, or a
 * latency-critical loop that cannot absorb cudaMalloc's implicit device
 * synchronisation. Everything a plan would allocate (descriptor copy, work
 * list, DFT tables, sample ring, error flag) lives in one file-scope device
 * array of MTB_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library
 * holds until exit; a configuration that needs more is rejected with
 * MTB_INVALID_ARG and the byte count in mtb_last_error(). The caller passes
 * the inputs and outputs exactly as for mtb_yee2d_plan_create (struct,
 * regions, groups; amp_col 0 is the only coefficient column) plus `parity`,
 * the ping-pong buffer holding the current state; after the call the state is
 * in buffer parity ^ (k & 1). The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and sets kernel attributes, so make
 * it before any stream capture; that set-up is guarded by a lock, so host
 * threads may make first calls concurrently. The cached address belongs to
 * the device's primary context: after cudaDeviceReset the entry point must
 * not be called on that device again (unsupported). Every call shares the
 * one array: calls whose work overlaps on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.
 * Before any step kernel runs, the call checks on the device each source
 * list's row_ptr (starts at 0, ends at n, never decreases), the column order
 * within each row and the line samples, and waits for that verdict on
 * `stream`: a rejected call (MTB_INVALID_ARG) leaves the caller's fields,
 * CPML memory and accumulators untouched. The call also waits for its work
 * on `stream` before returning (it reads back the bounded-wait error flag). */
#define MTB_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
int mtb_yee2d_run_noalloc(const mtb_yee2d_struct *s, const mtb_dft_region *regions,
                          int32_t n_regions, const mtb_phase_group *groups,
                          int32_t n_groups, int64_t ring_slot_elems, int32_t ring_slots,
                          int32_t parity, int64_t t0, int32_t k, const double *coef_e,
                          const double *coef_h, void *stream);

/* Waits for the plan's work on `stream` and reports a bounded device wait
 * that expired in any earlier run (MTB_DEVICE_TIMEOUT) -- the kernels never
 * spin forever; a wait that gives up sets this flag and the step returns. */
int mtb_yee2d_check(mtb_yee2d_plan *plan, void *stream);

/* Number of kernel launches the last mtb_yee2d_run issued. */
int64_t mtb_yee2d_last_launches(const mtb_yee2d_plan *plan);

/* Opt-in device timing: with enable = 1 every later run records a CUDA
 * event pair around each step-kernel launch and each DFT-contraction launch
 * on its stream, and waits for them at its end; mtb_yee2d_timing returns the
 * summed device milliseconds and launch counts since timing was enabled. */
int mtb_yee2d_set_timing(mtb_yee2d_plan *plan, int32_t enable);
int mtb_yee2d_timing(const mtb_yee2d_plan *plan, double *step_ms, int64_t *step_launches,
                     double *dft_ms, int64_t *dft_launches);

void mtb_yee2d_plan_destroy(mtb_yee2d_plan *plan);

/* The plan's DFT sample ring: slot s (0 <= s < ring_slots) of the last run
 * holds the samples of that run's step s (ring + s * slot_elems), in the
 * layout the structures' ring_full / lines offsets describe. */
int mtb_yee2d_ring(const mtb_yee2d_plan *plan, float **ring, int64_t *slot_elems,
                   int32_t *ring_slots);

/* Copy samples out of the plan's ring after a run of n_slots <= ring_slots
 * steps (one flush): out[s * n_off + j] = ring[s * slot_elems + offsets[j]]
 * for s < n_slots (offsets and out are device arrays; an offset outside the
 * slot reads 0). This is the "stack" reduction of core/run.py:28-38 for
 * probes such as PointProbe (core/monitors.py:11-21): one value per step
 * instead of a running sum. */
int mtb_yee2d_ring_gather(const mtb_yee2d_plan *plan, const int64_t *offsets, int32_t n_off,
                          int32_t n_slots, float *out, void *stream);

/* ---------------------------------------------------------- 2D adjoint */
/* Discrete adjoint (reverse mode) of the TM and TE steps, the transpose of
 * core/stepper_tm.py:234-254 / core/stepper_te.py:178-190 with CPML and PEC
 * walls, electric conductivity, magnetic conductivity and permeability, and
 * dispersive ADE poles (TM and TE) and of the DFT / flux
 * sampling
 * (core/monitors.py:24-155): what torch autograd computes through the
 * reference's run_tm / run_te (core/run.py:43-126).
 *
 * Adjoint state (box layout of the structure, nx x pitch floats each, one
 * buffer per array), holding on entry d J / d (state after the last step of
 * the call) and on return d J / d (state before its first step):
 *   TM: g[0] Ez, g[1] Hx, g[2] Hy, g[3] Dz;  TE: g[0] Hz, g[1] Ex, g[2] Ey,
 *   g[3] Dx, g[4] Dy;  g_psi[0..3] as mtb_yee2d_struct psi.
 * tmp[0..3]: scratch of the same size. g_eps accumulates d J / d eps (box
 * layout; the caller zeroes it once): TM g_eps[0] = eps_inf; TE g_eps[0] =
 * eps_x (Ex nodes), g_eps[1] = eps_y (Ey nodes). */
typedef struct mtb_adj2d_buffers {
    float *g[5];
    float *g_psi[4];
    float *tmp[4];
    float *g_eps[2];
    /* With dispersive poles: d J / d P(n) (g_pol[0]) and d J / d P(n-1)
     * (g_pol[1]), n_poles planes of nx x pitch floats each (TM P on Ez, TE Px on
     * Ex); g_pol_y the same for TE's Py stack (n_poles_y planes); null otherwise */
    float *g_pol[2];
    float *g_pol_y[2];
    /* With a live on-plane H line (cut_y / cut_x 2: TM odd mirrors, Rotate2,
     * Rotate4): d J / d Hx0 (g_cut[0], nx floats) and d J / d Hy0 (g_cut[1], ny
     * floats), two buffers each (alternate reverse steps); zero at creation,
     * null otherwise */
    float *g_cut[2][2];
    /* With TM magnetic poles: d J / d B (g_b[0] Bx, g_b[1] By, box arrays) and
     * d J / d M(n), d J / d M(n-1) (g_mpol[c][0], g_mpol[c][1], n_mpoles planes
     * each); null otherwise */
    float *g_b[2];
    float *g_mpol[2][2];
} mtb_adj2d_buffers;

typedef struct mtb_yee2d_adjoint mtb_yee2d_adjoint;

/* `s` is the forward structure (its ring_full / lines give the sample
 * layout of the forward ring, slot size ring_slot_elems); `regions` are the
 * forward DFT regions with `acc` pointing at d J / d acc (read only). */
int mtb_yee2d_adjoint_create(const mtb_yee2d_struct *s, const mtb_adj2d_buffers *bufs,
                             const mtb_dft_region *regions, int32_t n_regions,
                             const mtb_phase_group *groups, int32_t n_groups,
                             int64_t ring_slot_elems, int32_t ring_slots,
                             mtb_yee2d_adjoint **out);
/* Reverse steps t0+k-1 .. t0 (k <= ring_slots). `rec` slot q (slot size
 * rec_slot_elems) holds the forward E of step t0+q (the ring of a forward
 * plan that ran these k steps with full-grid E samples): TM Ez after the step
 * at rec_offset[0] + box index; TE Ex, Ey of the step at rec_offset[0],
 * rec_offset[1]. */
int mtb_yee2d_adjoint_run(mtb_yee2d_adjoint *p, int64_t t0, int32_t k, const float *rec,
                          int64_t rec_slot_elems, const int64_t *rec_offset, void *stream);
int64_t mtb_yee2d_adjoint_last_launches(const mtb_yee2d_adjoint *p);
void mtb_yee2d_adjoint_destroy(mtb_yee2d_adjoint *p);

/* ---------------------------------------------------------------- 3D */

/* One 3D structure (State3D / Coeffs3D, CPML path, sigma = 0, no poles).
 * Box layout: every array nx x ny x zpitch floats, zpitch % 4 == 0,
 * zpitch >= nz; the component's reference array in the low corner.
 * E is stored (the functional stepper's primary), eps is cell-centred. */
typedef struct mtb_yee3d_struct {
    int32_t nx, ny, nz, zpitch;
    float dt, dx;
    int32_t point_sign;     /* +1 step_3d (adds), -1 lean (subtracts)       */
    int32_t pad_;
    float *f[6][2];         /* Ex Ey Ez Hx Hy Hz, ping-pong pairs           */
    const float *eps;       /* cell-centred eps (nx, ny, nz) in box layout  */
    /* CPML memory in box layout, order of core/stepper_3d.py:46-57:
     * Ez_y Ey_z Ex_z Ez_x Ey_x Ex_y Hz_y Hy_z Hx_z Hz_x Hy_x Hx_y */
    float *psi[12][2];
    /* (b, a) profiles: [axis][0] half nodes (n-1), [axis][1] integer nodes (n) */
    const float *prof_b[3][2];
    const float *prof_a[3][2];
    /* soft current: cells (i, j, k) on component src_comp, CSR over the
     * (i, j) rows (row_ptr has nx*ny+1 entries, row i*ny+j; col = k).
     * Point sources follow point_sign; mask sources always subtract
     * (core/stepper_3d.py:452-461). amp_col must be 0. */
    int32_t src_comp;
    int32_t src_is_point;
    mtb_cells src;
    /* plane samples: component `comp` at plane `index` normal to `axis`,
     * window [lo0, hi0) x [lo1, hi1) of the two in-plane axes (in order),
     * copied row-major to ring_off. */
    const int32_t *planes;  /* device int32[n_planes][8]:
                               comp, axis, index, lo0, hi0, lo1, hi1, unused */
    const int64_t *plane_ring_off; /* device int64[n_planes]               */
    int32_t n_planes;
    int32_t pad2_;
    /* conductive damping (core/stepper_3d.py:217-235 damp pairs from sigma_d /
     * sigma_b, applied at :375-437): per component (Ex Ey Ez Hx Hy Hz) the pair
     * (d1, d2) as box arrays, H' = d1 H - d2 curl E, E' = d1 E + d2 curl H / eps;
     * all null = the plain step (d1 = 1, d2 = dt). Split kernels only; the
     * fused kernel and the adjoint return MTB_UNSUPPORTED. */
    const float *damp[6][2];
    /* dispersive poles (core/stepper_3d.py:236-300; the functional stepper's
     * folded-D update): n_poles (<= MTB_MAX_POLES) box planes per E component
     * (Ex Ey Ez), plane k at k * nx * ny * zpitch. pol_p[c][2] ping-pong with the
     * fields: buffer `cur` P(n), the other P(n-1), overwritten with
     * P(n+1) = c1 P(n) + c2 P(n-1) + c3 E(n); c1, c2 per pole (host values),
     * c3 per cell. Split kernels and the adjoint. */
    int32_t n_poles;
    /* PMC walls instead of PEC on these axes (bit 0 x, 1 y, 2 z; core/stepper_3d.py
     * _term_pmc :99-121): the tangential E stays live at the wall and the curl term
     * that differentiates along the axis is zero there. The split and one-pass
     * kernels and the adjoint take it; the register-staged march refuses it. */
    int32_t pmc_axes;
    float *pol_p[3][2];
    const float *pol_c3[3];
    float pol_c1[MTB_MAX_POLES];
    float pol_c2[MTB_MAX_POLES];
} mtb_yee3d_struct;

typedef struct mtb_yee3d_plan mtb_yee3d_plan;

int mtb_yee3d_plan_create(const mtb_yee3d_struct *s,
                          const mtb_dft_region *regions, int32_t n_regions,
                          const mtb_phase_group *groups, int32_t n_groups,
                          int64_t ring_slot_elems, const mtb_tuning *tuning,
                          mtb_yee3d_plan **out);
int mtb_yee3d_run(mtb_yee3d_plan *plan, int64_t t0, int32_t k,
                  const double *coef, void *stream);
/* Error flag of the one-pass kernel (variant 3): MTB_DEVICE_TIMEOUT if one of
 * its bounded waits for a staged plane copy expired since the plan was made
 * (the steps of that launch are incomplete). Synchronises `stream`; call it
 * before trusting the state (the engine does when it exports fields). */
int mtb_yee3d_check(mtb_yee3d_plan *plan, void *stream);
/* x-slab decomposition (core/monitors_3d.py:192-210 run_3d split across
 * ranks along x). The plan holds planes [lo, hi) of a larger grid as its own
 * nx planes: its first plane is the left neighbour's last plane (a halo)
 * unless lo == 0, its last the right neighbour's first unless hi == the global
 * nx. set_slab restricts the updates to the plan's planes [own_lo, own_hi);
 * the halo planes are the caller's to fill. Split kernels only. */
int mtb_yee3d_set_slab(mtb_yee3d_plan *plan, int32_t own_lo, int32_t own_hi);
/* Half steps, so that a caller can exchange halo planes between the H and E
 * updates: begin stages steps t0 .. t0+k-1 (amplitudes coef[0..k-1] as in
 * mtb_yee3d_run); then per step half(0) = H(n+1/2) from E(n) (written to
 * the buffer mtb_yee3d_current() ^ 1) and half(1) = E(n+1), the plane
 * samples and the ring fold (the buffers flip). Same results as
 * mtb_yee3d_run of the k steps. */
int mtb_yee3d_begin(mtb_yee3d_plan *plan, int64_t t0, int32_t k, const double *coef,
                    void *stream);
int mtb_yee3d_half(mtb_yee3d_plan *plan, int32_t part, void *stream);
int32_t mtb_yee3d_current(const mtb_yee3d_plan *plan);
int64_t mtb_yee3d_last_launches(const mtb_yee3d_plan *plan);
int mtb_yee3d_set_timing(mtb_yee3d_plan *plan, int32_t enable);
int mtb_yee3d_timing(const mtb_yee3d_plan *plan, double *step_ms, int64_t *step_launches,
                     double *dft_ms, int64_t *dft_launches);
void mtb_yee3d_plan_destroy(mtb_yee3d_plan *plan);

/* ------------------------------------------------------- 3D adjoint */
/* Discrete adjoint of the 3D CPML step (core/stepper_3d.py:363-482) and of
 * the plane sampling (core/monitors_3d.py:70-189): the reverse sweep of the
 * reference's run_3d_adjoint (core/adjoint3d.py:56-115).
 *   g[0..5]   d J / d (Ex, Ey, Ez, Hx, Hy, Hz), box layout (nx x ny x zpitch)
 *   g_psi     d J / d psi (12, as mtb_yee3d_struct psi)
 *   tmp[0..14] scratch boxes; g_eps accumulates d J / d eps (cell-centred).
 *   g_pol[c][0] / g_pol[c][1]  with dispersive poles: d J / d P(n) and
 *              d J / d P(n-1) of E component c, n_poles box planes each (the
 *              layout of mtb_yee3d_struct.pol_p); null without poles. */
typedef struct mtb_adj3d_buffers {
    float *g[6];
    float *g_psi[12];
    float *tmp[15];
    float *g_eps;
    float *g_pol[3][2];
} mtb_adj3d_buffers;

typedef struct mtb_yee3d_adjoint mtb_yee3d_adjoint;

int mtb_yee3d_adjoint_create(const mtb_yee3d_struct *s, const mtb_adj3d_buffers *bufs,
                             const mtb_dft_region *regions, int32_t n_regions,
                             const mtb_phase_group *groups, int32_t n_groups,
                             int64_t ring_slot_elems, int32_t ring_slots,
                             mtb_yee3d_adjoint **out);
/* Reverse steps t0+k-1 .. t0 (k <= ring_slots). E component c (0..2) of
 * record slot q (0..k) is at rec + q * rec_slot_stride + c * rec_comp_stride
 * (box layout): slot 0 holds E before step t0, slot q the E after step
 * t0+q-1. */
int mtb_yee3d_adjoint_run(mtb_yee3d_adjoint *p, int64_t t0, int32_t k, const float *rec,
                          int64_t rec_comp_stride, int64_t rec_slot_stride, void *stream);
int64_t mtb_yee3d_adjoint_last_launches(const mtb_yee3d_adjoint *p);
void mtb_yee3d_adjoint_destroy(mtb_yee3d_adjoint *p);

/* ------------------------------------------------------------ layout */

/* Strided copy of an n0 x n1 x n2 block between a dense reference array
 * (strides s0, s1, 1 in elements) and a box array (strides b0, b1, 1).
 * mtb_pack writes box[i,j,k] = src[i,j,k] for the block and zero for the
 * rest of the box row range [0, b_rows) x [0, b1_extent); mtb_unpack copies
 * the block back. Both run on `stream`. */
int mtb_pack(const float *src, int64_t n0, int64_t n1, int64_t n2,
             int64_t s0, int64_t s1, float *box, int64_t box_n0,
             int64_t box_n1, int64_t box_n2, int64_t b0, int64_t b1,
             int64_t off0, int64_t off1, int64_t off2, void *stream);
int mtb_unpack(const float *box, int64_t n0, int64_t n1, int64_t n2,
               int64_t b0, int64_t b1, int64_t off0, int64_t off1,
               int64_t off2, float *dst, int64_t s0, int64_t s1, void *stream);
/* As mtb_unpack, dividing by a second box array of the same layout:
 * dst = box / den (E = D / eps when exporting a 2D state, the reference's
 * update_eh(E), core/stepper_tm.py:224-231). */
int mtb_unpack_ratio(const float *box, const float *den, int64_t n0, int64_t n1,
                     int64_t n2, int64_t b0, int64_t b1, int64_t off0,
                     int64_t off1, int64_t off2, float *dst, int64_t s0,
                     int64_t s1, void *stream);

/* Count entries of x (n floats) whose |x| > 0 where mask_row (per leading
 * index, n0 entries) and mask_col (per last index) are both zero -- used to
 * check CPML memory is zero outside the absorbing layers on import. */
int mtb_count_outside(const float *x, int64_t n0, int64_t n1, int64_t s0,
                      const uint8_t *active0, const uint8_t *active1,
                      int64_t *count_dev, void *stream);

/* ------------------------------------------------- FNO channel mixes */

/* The pointwise (1 x 1) layers of the Fourier neural operator of the surrogate
 * design loop, on the tcgen05 tensor cores (no counterpart in the reference):
 * BF16 operands, FP32 accumulation in TMEM. Tensors are NCHW float32 with
 * `pixels` = H * W (a multiple of 8) per channel; built shapes: cin = 64, cout
 * 64 or 128. All kernels run on `stream` and return at once; a bounded
 * tensor-core wait that expired is reported by mtb_fno_status.
 *
 * mtb_fno_mix:    z = W x + bias + s (bias [cout] and s [batch, cout, pixels]
 *                 optional), y = act ? GELU(z) : z (exact erf GELU); z is
 *                 stored when non-NULL. W is [cout, cin] row-major.
 * mtb_fno_mix_dx: dz = act ? dy * GELU'(z) : dy (stored when non-NULL),
 *                 dx = W^T dz.
 * mtb_fno_mix_dw: dw += dz x^T summed over images and pixels (dw [cout, cin],
 *                 accumulated: zero it first); dz and x 16-byte aligned. */
int mtb_fno_mix(const float *x, const float *w, const float *bias, const float *s, float *y,
                float *z, int32_t batch, int32_t cin, int32_t cout, int64_t pixels,
                int32_t act, void *stream);
int mtb_fno_mix_dx(const float *dy, const float *z, const float *w, float *dz, float *dx,
                   int32_t batch, int32_t cin, int32_t cout, int64_t pixels, int32_t act,
                   void *stream);
int mtb_fno_mix_dw(const float *dz, const float *x, float *dw, int32_t batch, int32_t cin,
                   int32_t cout, int64_t pixels, void *stream);
/* Waits for `stream`; MTB_DEVICE_TIMEOUT (and clears the flag) if a tensor-core
 * wait of an earlier FNO launch expired. */
int mtb_fno_status(void *stream);

/* ------------------------------------------------------------ misc */

const char *mtb_last_error(void);
int32_t mtb_abi_version(void);
/* sizeof of the ABI structs, for binding checks: 0 mtb_cells,
 * 1 mtb_line_sample, 2 mtb_yee2d_struct, 3 mtb_phase_group,
 * 4 mtb_dft_region, 5 mtb_tuning, 6 mtb_yee3d_struct, 7 mtb_adj2d_buffers,
 * 8 mtb_adj3d_buffers */
int64_t mtb_struct_size(int32_t which);
/* Kernels launched by this library since load (all entry points). */
int64_t mtb_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* MEEP_B200_H */
