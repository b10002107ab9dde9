/*
 * castro_b200.h -- C-ABI of the B200 CTU hydro advance (libcastro_b200.so).
 *
 * Two layers:
 *
 * 1. The reference's Fortran entry points, Source/Castro_F.H:11-161, with the
 *    same names, argument order and meaning.  Each takes a whole box [lo,hi]
 *    and launches one kernel over it on the library stream; arrays are device
 *    (or managed) pointers in BL_FORT_FAB_ARG_3D form (pointer, lo[3], hi[3]),
 *    Fortran order, component slowest; lo/hi/dx pointers are host pointers.
 *    The reference calls these per zone from inside an AMReX device lambda
 *    (Source/Castro.H:23-27); a host replacing the Fortran objects calls them
 *    once per box instead.  Like the reference they
 *    return void; errors are reported through castro_last_error().
 *
 * 2. Coarse entry points with no reference counterpart at the ABI level but
 *    replacing whole host routines: castro_construct_hydro_source_box
 *    (Castro::construct_hydro_source's MFIter body, Source/Castro_hydro.cpp:31-397)
 *    and the castro_sim_* family (Castro::advance / estTimeStep /
 *    computeNewDt / post_timestep and the Amr coarse step loop,
 *    Source/Castro_advance.cpp:12-100, Source/Castro.cpp:162-426,
 *    Source/main.cpp:127-168), in a plain per-box form and a batched form
 *    that advances every box of every instance with one fused kernel
 *    sequence per step.
 *
 * Species: the reference fixes nspec = 13 at compile time
 * (Source/network.F90:7); this library takes the network at run time through
 * castro_network_init and supports nspec = 2 and nspec = 13.
 */
#ifndef CASTRO_B200_H
#define CASTRO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CASTRO_MAX_SPEC 13

/* ------------------------------------------------------------------------- */
/* Library state and errors (no reference counterpart: the Fortran returns    */
/* void and aborts through amrex_error)                                       */
/* ------------------------------------------------------------------------- */
enum {
    CASTRO_OK = 0,
    CASTRO_ERR_CUDA = 1,        /* a CUDA call failed; see castro_error_string */
    CASTRO_ERR_NO_TABLE = 2,    /* eos_init has not succeeded */
    CASTRO_ERR_TABLE_IO = 3,    /* helm_table.dat missing or malformed */
    CASTRO_ERR_NSPEC = 4,       /* network size other than 2 or 13 */
    CASTRO_ERR_ARG = 5,         /* invalid argument */
    CASTRO_ERR_EOS = 6,         /* EOS Newton iteration did not converge */
    CASTRO_ERR_IO = 7,          /* a checkpoint or plotfile could not be read or written */
    CASTRO_ERR_TIMEOUT = 8      /* a device-side wait ran out of its iteration limit; the step is void */
};
int         castro_last_error(void);          /* sticky: first error since castro_clear_error */
void        castro_clear_error(void);
const char* castro_error_string(void);
int         castro_version(void);
/* stream used by every launch (a cudaStream_t); default is the legacy stream 0 */
void        castro_set_stream(void* stream);
void*       castro_get_stream(void);
/* 1 when the library was built with CASTRO_EXACT (no FMA contraction, the
 * reference's operation order everywhere) */
int         castro_exact_build(void);

/* ------------------------------------------------------------------------- */
/* Source/Castro_F.H:11-17                                                    */
/* ------------------------------------------------------------------------- */
void network_init(void);                      /* Castro_F.H:11: the 13-species network of Source/network.F90 */
void network_finalize(void);                  /* Castro_F.H:13 */
/* run-time network (replaces the compile-time parameters of Source/network.F90:7-19) */
int  castro_network_init(int nspec, const double* aion, const double* zion);
int  castro_nspec(void);
/* Keep the packed EOS table (13.9 MB) resident in L2 with a persisting
 * access-policy window on the streams of sims created afterwards (default on;
 * 0 switches it off for sims created later).  No reference counterpart: the
 * reference reads the table through ordinary loads.  The L2 set-aside belongs
 * to this process's CUDA context and eos_finalize puts the previous value back. */
void castro_set_table_l2_window(int on);
/* Batched sims (2 species) created afterwards form the cross fluxes and the
 * final fluxes of the CTU step (Source/Castro_hydro.cpp:228-359) in one kernel
 * per column tile, marching in z with the cross-flux records in shared memory,
 * instead of two kernels passing them through HBM; results are the same bit for
 * bit.  Off by default: on B200 the fused kernel, at lower occupancy than the
 * two kernels and with a block-wide barrier per phase and plane, is slower.  No
 * reference counterpart. */
void castro_set_column_tiles(int on);
int  castro_column_tiles(void);

/* Option, off by default (no counterpart in the reference): the interface
 * pressure in the normal momentum flux of compute_flux, flx(im1) = rho u u + p,
 * as full Castro has it in Cartesian geometry.  The reference's compute_flux
 * (Source/riemann.F90:306-308) and consup (Source/Castro_hydro_nd.F90:344-441)
 * put no pressure gradient in the momentum equation, so its blasts expand far
 * slower than a Sedov-Taylor blast; with the option the same kernels follow the
 * Sedov-Taylor solution.  Library-wide (every kernel, the adjoint included);
 * the call waits for the kernels already queued on the device, which run with
 * the old setting.  The oracle's oracle_set_momentum_flux_pressure is its
 * counterpart. */
void castro_set_momentum_flux_pressure(int on);
int  castro_momentum_flux_pressure(void);

/* Option, off by default: Coulomb corrections in the EOS.  The reference's
 * eos.F90 has none; its 2017 runs used them ("Initializing Helmholtz EOS and
 * using Coulomb corrections", scaling/summitdev_20171020/1.out:14).  The ion
 * plasma's excess energy and pressure in a uniform electron background from
 * the fits of Yakovlev & Shalybkov (1989), as the Helmholtz EOS applies them
 * (Timmes & Swesty 2000): added to p, e and their density and temperature
 * derivatives wherever the EOS is evaluated, unless the totals would turn
 * non-positive there.  The forward paths only: the adjoint (castro_adj_*, the
 * *_adj routines that call the EOS) refuses to run with it (CASTRO_ERR_ARG).
 * The call waits for the kernels already queued on the device.  Each launch
 * reads the setting (a sim captures its step again when it changed); a CUDA
 * graph a caller captured around the per-box entry points keeps the setting it
 * was captured with.  The oracle's oracle_set_coulomb_corrections is its
 * counterpart. */
void castro_set_coulomb_corrections(int on);
int  castro_coulomb_corrections(void);

void eos_init(void);                          /* Castro_F.H:15: reads ./helm_table.dat (or $CASTRO_HELM_TABLE), eos.F90:580-734 */
void eos_finalize(void);                      /* Castro_F.H:17 */
int  castro_eos_init_path(const char* path);  /* eos_init with an explicit table path; returns an error code */

/* ------------------------------------------------------------------------- */
/* Per-routine entry points, Source/Castro_F.H:19-161                         */
/* ------------------------------------------------------------------------- */
/* Castro_F.H:19-23 -> Castro_hydro_nd.F90:73 */
void ctoprim(const int* lo, const int* hi,
             const double* u, const int* u_lo, const int* u_hi,
             const double* q, const int* q_lo, const int* q_hi,
             const double* qaux, const int* qa_lo, const int* qa_hi);
/* Castro_F.H:25-27 -> Castro_nd.F90:69 */
void enforce_minimum_density(const int* lo, const int* hi, double* state, const int* s_lo, const int* s_hi);
/* Castro_F.H:29-31 -> Castro_nd.F90:129 */
void normalize_species(const int* lo, const int* hi, double* state, const int* s_lo, const int* s_hi);
/* Castro_F.H:33-35 -> Castro_nd.F90:164 */
void reset_internal_e(const int* lo, const int* hi, double* state, const int* s_lo, const int* s_hi);
/* Castro_F.H:37-39 -> Castro_nd.F90:253 */
void compute_temp(const int* lo, const int* hi, double* state, const int* s_lo, const int* s_hi);
/* Coarse entry point for Castro::clean_state on one box (Source/Castro.cpp:563-591):
 * enforce_minimum_density, normalize_species, reset_internal_e and compute_temp
 * in one launch instead of four.  Each of the four is pointwise, so applying
 * them zone by zone gives the four calls' results bit for bit. */
void castro_clean_state(const int* lo, const int* hi, double* state, const int* s_lo, const int* s_hi);
/* Castro_F.H:41-45 -> timestep.F90:12; dt is a device/managed double lowered atomically */
void estdt(const int* lo, const int* hi, const double* state, const int* s_lo, const int* s_hi,
           const double* dx, double* dt);
/* MultiFab::Saxpy(S_new, dt, hydro_source) of Source/Castro_advance.cpp:74 (an
 * AMReX call, not a Castro_F.H routine): u[m] = u[m] + dt * src[m] over n
 * doubles of device memory, on the library stream */
void castro_saxpy(double* u, const double* src, long long n, double dt);

/* The AMR pieces (no counterpart in the reference's own code, which hands them to
 * AMReX): Castro::reflux's flux register (Source/Castro.cpp:451-483) and
 * Castro::avgDown (:486-504).  Fluxes are store_flux's dt * F * A on face boxes.
 * For the coarse faces [flo, fhi] (coarse indices, normal direction dir) on one
 * side of a fine patch refined by `ratio`:
 *   crse_init: reg = -crse_flux;
 *   fine_add:  reg += the sum of the ratio^2 fine face fluxes over each coarse face
 *              (call once per fine substep);
 *   reflux:    the coarse zone on `side` of each face (0: below, the patch above;
 *              1: above) gets -reg / volume (side 0) or +reg / volume (side 1).
 * average_down: each coarse zone of [clo, chi] = the mean of its ratio^3 fine zones.
 * A zone or face the call would read or write outside its array's box: nothing
 * is launched and castro_last_error() is CASTRO_ERR_ARG. */
void castro_flux_register_crse_init(const int* flo, const int* fhi, double* reg, const int* r_lo, const int* r_hi,
                                    const double* crse_flux, const int* c_lo, const int* c_hi, int ncomp);
void castro_flux_register_fine_add(const int* flo, const int* fhi, int dir, double* reg, const int* r_lo,
                                   const int* r_hi, const double* fine_flux, const int* f_lo, const int* f_hi,
                                   int ncomp, int ratio);
void castro_flux_register_reflux(const int* flo, const int* fhi, int dir, int side, double* state, const int* s_lo,
                                 const int* s_hi, const double* reg, const int* r_lo, const int* r_hi, int ncomp,
                                 double volume);
void castro_average_down(const int* clo, const int* chi, double* crse, const int* c_lo, const int* c_hi,
                         const double* fine, const int* f_lo, const int* f_hi, int ncomp, int ratio);
/* Castro_F.H:47-53 -> Castro_hydro_nd.F90:301 */
void store_flux(const int* lo, const int* hi,
                double* flux_out, const int* fo_lo, const int* fo_hi,
                double* flux_in, const int* fi_lo, const int* fi_hi,
                double* area, const int* a_lo, const int* a_hi, const double dt);
/* Castro_F.H:55-71 -> Castro_hydro_nd.F90:344 (consup) */
void fill_hydro_source(const int* lo, const int* hi,
                       const double* state, const int* s_lo, const int* s_hi,
                       const double* q, const int* q_lo, const int* q_hi,
                       double* source, const int* sr_lo, const int* sr_hi,
                       const double* flux0, const int* f0_lo, const int* f0_hi,
                       const double* flux1, const int* f1_lo, const int* f1_hi,
                       const double* flux2, const int* f2_lo, const int* f2_hi,
                       const double* qe0, const int* qe0_lo, const int* qe0_hi,
                       const double* qe1, const int* qe1_lo, const int* qe1_hi,
                       const double* qe2, const int* qe2_lo, const int* qe2_hi,
                       const double* area0, const int* a0_lo, const int* a0_hi,
                       const double* area1, const int* a1_lo, const int* a1_hi,
                       const double* area2, const int* a2_lo, const int* a2_hi,
                       const double* volume, const int* v_lo, const int* v_hi,
                       const double* dx, const double dt);
/* Castro_F.H:73-76 -> Castro_hydro_nd.F90:248 */
void normalize_species_fluxes(const int* lo, const int* hi, double* flux, const int* f_lo, const int* f_hi);
/* Castro_F.H:78-84 -> Castro_hydro_nd.F90:174; idir is 1-based */
void apply_av(const int* lo, const int* hi, const int idir, const double* dx,
              double* div, const int* d_lo, const int* d_hi,
              double* Sborder, const int* s_lo, const int* s_hi,
              double* flux, const int* f_lo, const int* f_hi);
/* Castro_F.H:86-96 -> trans.F90:14 */
void trans1(const int* lo, const int* hi, const int idir1, const int idir2,
            const double* q2m, const int* q2m_lo, const int* q2m_hi,
            double* q2mo, const int* q2mo_lo, const int* q2mo_hi,
            const double* q2p, const int* q2p_lo, const int* q2p_hi,
            double* q2po, const int* q2po_lo, const int* q2po_hi,
            const double* qaux, const int* qa_lo, const int* qa_hi,
            const double* f1, const int* f1_lo, const int* f1_hi,
            const double* q1, const int* q1_lo, const int* q1_hi,
            const double cdtdx);
/* Castro_F.H:98-110 -> trans.F90:250 */
void trans2(const int* lo, const int* hi, const int idir1, const int idir2, const int idir3,
            const double* qm, const int* qm_lo, const int* qm_hi,
            double* qmo, const int* qmo_lo, const int* qmo_hi,
            const double* qp, const int* qp_lo, const int* qp_hi,
            double* qpo, const int* qpo_lo, const int* qpo_hi,
            const double* qaux, const int* qa_lo, const int* qa_hi,
            const double* fyz, const int* fyz_lo, const int* fyz_hi,
            const double* fzy, const int* fzy_lo, const int* fzy_hi,
            const double* qy, const int* qy_lo, const int* qy_hi,
            const double* qz, const int* qz_lo, const int* qz_hi,
            const double hdtdx, const double cdtdy, const double cdtdz);
/* Castro_F.H:112-121 -> riemann.F90:10 (riemanncg) */
void compute_flux(const int* lo, const int* hi,
                  const double* ql, const int* ql_lo, const int* ql_hi,
                  const double* qr, const int* qr_lo, const int* qr_hi,
                  double* flux, const int* fx_lo, const int* fx_hi,
                  double* q_int, const int* qi_lo, const int* qi_hi,
                  double* qe, const int* qe_lo, const int* qe_hi,
                  const double* qaux, const int* qa_lo, const int* qa_hi,
                  const int idir);
/* Castro_F.H:123-128 -> Castro_hydro_nd.F90:11 */
void divu(const int* lo, const int* hi, double* q, const int* q_lo, const int* q_hi,
          const double* dx, double* div, const int* d_lo, const int* d_hi);
/* Castro_F.H:130-140 -> ppm.F90:309 */
void trace_ppm(const int* lo, const int* hi, const int* vlo, const int* vhi, const int idir,
               const double* q, const int* q_lo, const int* q_hi,
               const double* qaux, const int* qa_lo, const int* qa_hi,
               double* qm, const int* qm_lo, const int* qm_hi,
               double* qp, const int* qp_lo, const int* qp_hi,
               const int* domlo, const int* domhi, const double* dx, const double dt);
/* Castro_F.H:142-146 -> Prob.F90:19; problem constants from castro_set_problem */
void initdata(const int* lo, const int* hi, double* state, const int* s_lo, const int* s_hi,
              const double* dx, const double* problo, const double* probhi);
/* Castro_F.H:148-153 -> Castro_nd.F90:301 */
void denerror(const int* lo, const int* hi, int8_t* tag, const int* tag_lo, const int* tag_hi,
              const double* den, const int* den_lo, const int* den_hi,
              const int8_t tagval, const int8_t clearval);
/* Castro_F.H:155-161 -> Castro_nd.F90:349; blast_mass/blast_radius are device doubles */
void calculate_blast_radius(const int* lo, const int* hi, double* state, const int* s_lo, const int* s_hi,
                            const double* dx, const double* problo, const double* probhi,
                            double* blast_mass, double* blast_radius, const double max_density);

/* ------------------------------------------------------------------------- */
/* Problem constants (Source/Prob.F90:11-15 plus the knobs of the benchmark   */
/* configurations)                                                            */
/* ------------------------------------------------------------------------- */
typedef struct {
    int    ambient_from_T;   /* 0: ambient e from EOS(rho,p) as Prob.F90:51-59; 1: from EOS(rho,T) */
    double dens_ambient;     /* g/cc */
    double p_ambient;        /* erg/cc (ambient_from_T == 0) */
    double T_ambient;        /* K (ambient_from_T == 1) */
    double exp_energy;       /* erg */
    double r_init;           /* cm */
    int    nsub;             /* subzones per dimension (Prob.F90:15: 10) */
    double X[CASTRO_MAX_SPEC];   /* initial mass fractions */
    double T_init;           /* UTEMP at init (Prob.F90:115: 1e9) */
    const double* pert;      /* optional device array over pert_lo..pert_hi: rho = dens_ambient*(1+pert_amp*pert) */
    int    pert_lo[3], pert_hi[3];
    double pert_amp;
} castro_problem;

/* Source/Prob.F90 defaults: rho=1e4, p=1e21, E=1e52, r=1.25e8, nsub=10, X1=1 */
void castro_problem_defaults(castro_problem* p);
int  castro_set_problem(const castro_problem* p);

/* ------------------------------------------------------------------------- */
/* Coarse entry point: construct_hydro_source for one box                     */
/* ------------------------------------------------------------------------- */
/* Castro::construct_hydro_source's body for one box (Source/Castro_hydro.cpp:31-397),
 * fused: Sborder (grow(box,4), NVAR comps, already cleaned) -> source on the box
 * (accumulated into 'source', which the caller zeroes like hydro_source.setVal(0)).
 * fluxes_out[d] (optional, may be NULL): dt*F*A on the faces of the box
 * (store_flux).  Runs on the stream of castro_set_stream.  Uses library-
 * managed scratch: one device array per (device, stream), up to 16 streams per
 * device, grown to the largest box seen on that stream so far; a call for a
 * box larger than every earlier one on its stream (or the first call of a
 * 17th stream) synchronizes the device and allocates (so do not capture such a
 * call in a CUDA graph), and every other call allocates nothing, whatever the
 * mix of box shapes.  Calls on one stream are ordered by it; calls on
 * different streams may overlap, as an AMReX MFIter loop's do. */
int castro_construct_hydro_source_box(const int* lo, const int* hi,
                                      const double* sborder, const int* sb_lo, const int* sb_hi,
                                      double* source, const int* sr_lo, const int* sr_hi,
                                      double* const* fluxes_out, const int* fo_lo3x3, const int* fo_hi3x3,
                                      const int* domlo, const int* domhi, const double* dx, double dt);

/* castro_construct_hydro_source_box without any device allocation.  No
 * counterpart in the reference.  For callers that cannot allocate device
 * memory while they advance a box: hosts that give out all device memory from
 * their own pool reserved at start-up, and hosts that must not call cudaMalloc
 * inside the time step because it synchronizes the device.  Same arguments,
 * meaning and result as castro_construct_hydro_source_box; its scratch lives in
 * one static device array of 18 MiB inside the library (held by every GPU that
 * loads the library until the process exits), which fits a box of at most
 * 16^3 zones with 13 species or 21^3 zones with 2 species; larger boxes are
 * rejected with CASTRO_ERR_ARG before anything is launched.  The first call
 * on each device (and species count) looks up the array's device address
 * (cudaGetSymbolAddress) and sets the Riemann kernels' shared-memory limits,
 * once, even when host threads make that first call together; make it before
 * any stream capture.  Later calls make no CUDA runtime call but the kernel
 * launches.  Every call shares the array and overwrites it: calls that overlap
 * on the GPU (two streams, two host threads) race and must be serialized by
 * the caller.  Kernels launch on
 * the library stream (castro_set_stream); allocates neither device nor host
 * memory on its success path. */
int castro_construct_hydro_source_box_noalloc(const int* lo, const int* hi,
                                              const double* sborder, const int* sb_lo, const int* sb_hi,
                                              double* source, const int* sr_lo, const int* sr_hi,
                                              double* const* fluxes_out, const int* fo_lo3x3, const int* fo_hi3x3,
                                              const int* domlo, const int* domhi, const double* dx, double dt);

/* ------------------------------------------------------------------------- */
/* Simulation driver: one level per instance, many instances per sim          */
/* ------------------------------------------------------------------------- */
typedef struct castro_sim castro_sim;

enum { CASTRO_BC_PERIODIC = 0, CASTRO_BC_OUTFLOW = 1 };
enum { CASTRO_MODE_PLAIN = 0,      /* per-box launches of the per-routine kernels, reference call sequence */
       CASTRO_MODE_BATCHED = 1,    /* fused kernels over every box of every instance, CUDA-graph replay */
       CASTRO_MODE_PLAIN_BOX = 2,  /* the reference call sequence per box, each box's hydro source from
                                    * castro_construct_hydro_source_box (what a Castro host calling the
                                    * coarse entry point from its MFIter loop runs) */
       CASTRO_MODE_PERSISTENT = 3 };/* the batched step as ONE cooperative launch: resident CTAs pull the
                                    * work items of every box of every instance from a device queue per
                                    * stage, grid barriers between stages with bounded waits, the next dt
                                    * formed in the epilogue */

typedef struct {
    int dom_lo[3], dom_hi[3];
    double problo[3], probhi[3];
    int bc;                       /* CASTRO_BC_* */
    int nbox;
    const int* box_lo;            /* 3*nbox, global indices */
    const int* box_hi;            /* 3*nbox */
    castro_problem prob;
    double stop_time;             /* < 0: none (Source/main.cpp:66 default is 0.01) */
} castro_instance_desc;

/* Creates the sim; NULL with CASTRO_ERR_ARG when an instance's domain is empty,
 * its zones are not cubic (the reference aborts on dx != dy != dz,
 * Source/Castro.cpp:95-100), its boundary condition is unknown, or its boxes are
 * empty, leave the domain, overlap or leave a gap: nothing is allocated then. */
castro_sim* castro_sim_create(int ninst, const castro_instance_desc* desc, int mode);
void   castro_sim_destroy(castro_sim* sim);
int    castro_sim_nbox(const castro_sim* sim, int inst);
/* number of doubles of box b's state FAB (valid box x NVAR) */
size_t castro_sim_box_size(const castro_sim* sim, int inst, int b);
/* device pointer of box b's state FAB (Fortran order, NVAR comps) */
double* castro_sim_box_state(castro_sim* sim, int inst, int b);
int    castro_sim_init_data(castro_sim* sim);
/* copy all boxes' state of every instance from/to one host buffer (instances
 * in order, boxes in order, each FAB contiguous); async on the library stream */
int    castro_sim_upload(castro_sim* sim, const double* host);
int    castro_sim_download(castro_sim* sim, double* host);
size_t castro_sim_total_size(const castro_sim* sim);
/* one Amr coarse step for every instance (dt choice, advance, post_timestep) */
int    castro_sim_step(castro_sim* sim);
int    castro_sim_run(castro_sim* sim, int nsteps);
/* host <-> device whole-run call: upload 'host_in', nsteps coarse steps,
 * download into 'host_out' (may alias host_in) */
int    castro_sim_run_host(castro_sim* sim, const double* host_in, int nsteps, double* host_out);
/* waits for the sim's stream; also reports, as CASTRO_ERR_EOS, EOS Newton
 * solves that hit their 100-iteration limit since the sim's last sync (a
 * non-finite or unphysical state: silent in the reference) */
int    castro_sim_sync(castro_sim* sim);
double castro_sim_time(castro_sim* sim, int inst);
double castro_sim_dt(castro_sim* sim, int inst);
int    castro_sim_steps(castro_sim* sim, int inst);
/* estTimeStep on the current state of instance inst (cfl included) */
double castro_sim_est_time_step(castro_sim* sim, int inst);
/* blast radius diagnostic of Source/Castro.cpp:371-424, cm */
double castro_sim_blast_radius(castro_sim* sim, int inst, double* blast_mass);
/* AMReX native plotfile of instance inst in directory dir (Header,
 * Level_0/Cell_H, Level_0/Cell_D_00000; one FAB per box of its BoxArray),
 * readable by AMReX tools -- the layout Amr::writePlotFile produces (the
 * reference never writes one by default: Source/main.cpp sets no plot_int) */
int    castro_sim_write_plotfile(castro_sim* sim, int inst, const char* dir);
/* Checkpoint / restart (the reference's State_Type checkpoint,
 * Source/Castro_setup.cpp:50-53, in a format of this library's own): dir/Header
 * (text: nspec, per instance its domain, BoxArray, time, completed steps, last dt
 * and stop time as exact hexadecimal floats) and dir/State_<n> (instance n's box
 * FABs, raw doubles in the castro_sim_download layout).  Reading needs a sim of
 * the same species count, domains and BoxArrays (CASTRO_ERR_ARG otherwise) and
 * checks the files completely before installing anything (CASTRO_ERR_IO); the
 * run then continues bit for bit as if it had not stopped, in any mode. */
int    castro_sim_write_checkpoint(castro_sim* sim, const char* dir);
int    castro_sim_read_checkpoint(castro_sim* sim, const char* dir);
/* CASTRO_MODE_PERSISTENT: the limit of every grid-barrier wait, in polls of
 * about 64 ns (default 2^24, ~1 s), after which the step ends with
 * CASTRO_ERR_TIMEOUT at the next castro_sim_sync.  Fault-injection hook for
 * tests: when extra > 0 the barrier after stage 'stage' (0 front ... 6 riemann3)
 * waits for 'extra' more CTAs than exist, so its wait must run out.  No
 * reference counterpart. */
int    castro_sim_set_wait_limit(castro_sim* sim, long long polls, int stage, int extra);
/* the CUDA stream (cudaStream_t) every launch of this sim is issued on */
void*  castro_sim_stream(castro_sim* sim);
/* batched mode: one step with a CUDA event around each of the fused kernels
 * (no graph); ms[k] receives the duration of kernel k and names[k] its name;
 * returns the number of kernels (at most 16) */
int    castro_sim_profile_step(castro_sim* sim, double* ms, const char** names);
/* kernel launches issued by the last castro_sim_step (graph nodes for the batched mode) */
int    castro_sim_launches_per_step(const castro_sim* sim);
/* EOS Newton solves that hit their iteration limit since the sim was created */
long long castro_sim_eos_failures(castro_sim* sim);

/* FP64 fused-multiply-add throughput of the current device in TFLOP/s,
 * measured with a dependent-chain DFMA kernel over every SM (roofline
 * denominator of the FP64 kernels; no reference counterpart) */
double castro_measure_fp64_tflops(void);

/* the mini-app driver with the reference's command-line keys (Source/main.cpp) */
int castro_main(int argc, char** argv);

/* ------------------------------------------------------------------------- */
/* Reverse mode (adjoint).  No counterpart in the reference: each entry point  */
/* is the adjoint of the Castro_F.H routine it is named after, over the same   */
/* [lo,hi] and FAB conventions.  Given the routine's primal inputs and the     */
/* adjoint of its outputs (suffix b), it ACCUMULATES J^T * (output adjoint)     */
/* into the adjoint of its inputs.  Branch decisions (limiters, floors, the    */
/* Riemann sampling) follow the forward at the given inputs.  Components with  */
/* no consumer on the hydro path carry no adjoint: QGAME and QTEMP of face      */
/* states, the Riemann interface state q_int, and UTEMP (a Newton initial      */
/* guess only).  Scatters into shared arrays use FP64 atomics.                 */
/* ------------------------------------------------------------------------- */
/* Castro_F.H:19-23 */
void ctoprim_adj(const int* lo, const int* hi, const double* u, const int* u_lo, const int* u_hi,
                 const double* qb, const int* qb_lo, const int* qb_hi, const double* qab, const int* qab_lo,
                 const int* qab_hi, double* ub, const int* ub_lo, const int* ub_hi);
/* Castro::clean_state (enforce_minimum_density, normalize_species,
 * reset_internal_e, compute_temp; Castro_F.H:25-39) on one FAB: u is the state
 * BEFORE cleaning; ub holds the adjoint of the cleaned state on entry and of u
 * on exit */
void clean_state_adj(const int* lo, const int* hi, const double* u, const int* u_lo, const int* u_hi, double* ub,
                     const int* ub_lo, const int* ub_hi);
/* Castro_F.H:123-128 */
void divu_adj(const int* lo, const int* hi, const double* dx, const double* divb, const int* d_lo, const int* d_hi,
              double* qb, const int* q_lo, const int* q_hi);
/* Castro_F.H:130-140 (uflatten included); dtb (device, may be NULL) += d/d(dt) */
void trace_ppm_adj(const int* lo, const int* hi, const int* vlo, const int* vhi, const int idir,
                   const double* q, const int* q_lo, const int* q_hi, const double* qaux, const int* qa_lo,
                   const int* qa_hi, const double* qmb, const int* qm_lo, const int* qm_hi, const double* qpb,
                   const int* qp_lo, const int* qp_hi, double* qb, const int* qb_lo, const int* qb_hi, double* qab,
                   const int* qab_lo, const int* qab_hi, const double* dx, const double dt, double* dtb);
/* Castro_F.H:112-121: fluxb / qeb are the adjoints of flux and qgdnv */
void compute_flux_adj(const int* lo, const int* hi, const double* ql, const int* ql_lo, const int* ql_hi,
                      const double* qr, const int* qr_lo, const int* qr_hi, const double* qaux, const int* qa_lo,
                      const int* qa_hi, const double* fluxb, const int* fx_lo, const int* fx_hi, const double* qeb,
                      const int* qe_lo, const int* qe_hi, double* qlb, const int* qlb_lo, const int* qlb_hi,
                      double* qrb, const int* qrb_lo, const int* qrb_hi, double* qab, const int* qab_lo,
                      const int* qab_hi, const int idir);
/* Castro_F.H:86-96; cdtdxb (device, may be NULL) += d/d(cdtdx) */
void trans1_adj(const int* lo, const int* hi, const int idir1, const int idir2,
                const double* q2m, const int* q2m_lo, const int* q2m_hi, const double* q2p, const int* q2p_lo,
                const int* q2p_hi, const double* qaux, const int* qa_lo, const int* qa_hi, const double* f1,
                const int* f1_lo, const int* f1_hi, const double* q1, const int* q1_lo, const int* q1_hi,
                const double cdtdx, const double* q2mob, const int* q2mob_lo, const int* q2mob_hi,
                const double* q2pob, const int* q2pob_lo, const int* q2pob_hi, double* q2mb, const int* q2mb_lo,
                const int* q2mb_hi, double* q2pb, const int* q2pb_lo, const int* q2pb_hi, double* qab,
                const int* qab_lo, const int* qab_hi, double* f1b, const int* f1b_lo, const int* f1b_hi, double* q1b,
                const int* q1b_lo, const int* q1b_hi, double* cdtdxb);
/* Castro_F.H:98-110 (hdtdx unused, as in the forward); cdtdyb/cdtdzb (device, may be NULL) */
void trans2_adj(const int* lo, const int* hi, const int idir1, const int idir2, const int idir3,
                const double* qm, const int* qm_lo, const int* qm_hi, const double* qp, const int* qp_lo,
                const int* qp_hi, const double* qaux, const int* qa_lo, const int* qa_hi, const double* fyz,
                const int* fyz_lo, const int* fyz_hi, const double* fzy, const int* fzy_lo, const int* fzy_hi,
                const double* qy, const int* qy_lo, const int* qy_hi, const double* qz, const int* qz_lo,
                const int* qz_hi, const double cdtdy, const double cdtdz, const double* qmob, const int* qmob_lo,
                const int* qmob_hi, const double* qpob, const int* qpob_lo, const int* qpob_hi, double* qmb,
                const int* qmb_lo, const int* qmb_hi, double* qpb, const int* qpb_lo, const int* qpb_hi, double* qab,
                const int* qab_lo, const int* qab_hi, double* fyzb, const int* fyzb_lo, const int* fyzb_hi,
                double* fzyb, const int* fzyb_lo, const int* fzyb_hi, double* qyb, const int* qyb_lo,
                const int* qyb_hi, double* qzb, const int* qzb_lo, const int* qzb_hi, double* cdtdyb, double* cdtdzb);
/* Castro_F.H:78-84: the flux adjoint passes through unchanged (flux += av) */
void apply_av_adj(const int* lo, const int* hi, const int idir, const double* dx, const double* div, const int* d_lo,
                  const int* d_hi, const double* sb, const int* s_lo, const int* s_hi, const double* fluxb,
                  const int* f_lo, const int* f_hi, double* divb, const int* db_lo, const int* db_hi, double* sbb,
                  const int* sbb_lo, const int* sbb_hi);
/* Castro_F.H:73-76: flux is the flux BEFORE normalization; fluxb in/out */
void normalize_species_fluxes_adj(const int* lo, const int* hi, const double* flux, const int* f_lo, const int* f_hi,
                                  double* fluxb, const int* fb_lo, const int* fb_hi);
/* Castro_F.H:55-71 */
void fill_hydro_source_adj(const int* lo, const int* hi, const double* sourceb, const int* sr_lo, const int* sr_hi,
                           const double* qe0, const int* qe0_lo, const int* qe0_hi,
                           const double* qe1, const int* qe1_lo, const int* qe1_hi,
                           const double* qe2, const int* qe2_lo, const int* qe2_hi,
                           const double* area0, const int* a0_lo, const int* a0_hi,
                           const double* area1, const int* a1_lo, const int* a1_hi,
                           const double* area2, const int* a2_lo, const int* a2_hi,
                           const double* volume, const int* v_lo, const int* v_hi, const double* dx,
                           double* flux0b, const int* f0_lo, const int* f0_hi,
                           double* flux1b, const int* f1_lo, const int* f1_hi,
                           double* flux2b, const int* f2_lo, const int* f2_hi,
                           double* qe0b, const int* qe0b_lo, const int* qe0b_hi,
                           double* qe1b, const int* qe1b_lo, const int* qe1b_hi,
                           double* qe2b, const int* qe2b_lo, const int* qe2b_hi);

/* Gradient of a Sedov run (one instance, one GPU).  The forward is initdata
 * plus nsteps coarse steps (computeNewDt, Castro::advance, post_timestep) over
 * the instance's domain as one box (the result does not depend on the
 * BoxArray); the objective is the kinetic energy in the spherical shell
 * r0 <= r / (probhi - problo) <= r1 about the domain centre (default 0.3-0.4).
 * The reverse sweep keeps a checkpoint every checkpoint_interval steps and
 * recomputes each segment; the time step's dependence on the state (CFL
 * reduction, 1.1x growth limit, stop-time clamp) is included.
 * desc->prob.pert (optional) must stay valid until the object is destroyed. */
typedef struct castro_adj castro_adj;
castro_adj* castro_adj_create(const castro_instance_desc* desc, int nsteps, int checkpoint_interval);
/* The same with two more choices, for domains whose per-step arrays do not fit
 * the device whole: slab_nz > 0 reverses every step slab by slab (z-slabs of
 * slab_nz zones, which must divide the domain's z extent): each slab recomputes
 * its forward from the domain's state with its true ghost zones, reverses it
 * seeded by the slab's part of the state adjoint, and adds its Sborder adjoint
 * into the domain's, so only one slab's intermediates and adjoints are held
 * (the states, checkpoints and state adjoints stay domain-sized).  first_step
 * > 0 differentiates only steps first_step .. nsteps-1: the forward runs the
 * earlier steps without recording, castro_adj_backward returns zero for the
 * problem parameters, and castro_adj_initial_adjoint gives dJ/dV at first_step.
 * castro_adj_create(desc, n, k) is castro_adj_create_window(desc, n, k, 0, 0).
 * No reference counterpart. */
castro_adj* castro_adj_create_window(const castro_instance_desc* desc, int nsteps, int checkpoint_interval,
                                     int slab_nz, int first_step);
void   castro_adj_destroy(castro_adj* adj);
/* new problem constants (energy, ambient density, perturbation ...) for the next forward */
int    castro_adj_set_problem(castro_adj* adj, const castro_problem* prob);
int    castro_adj_set_shell(castro_adj* adj, double r0, double r1);
/* forward run; *J receives the objective */
int    castro_adj_forward(castro_adj* adj, double* J);
/* reverse sweep after castro_adj_forward: dJ/d(exp_energy), dJ/d(dens_ambient)
 * and, if dJ_dpert is non-NULL (device array shaped like prob.pert), dJ/dpert
 * accumulated into it */
int    castro_adj_backward(castro_adj* adj, double* dJ_dE, double* dJ_drho, double* dJ_dpert);
double castro_adj_dt(const castro_adj* adj, int step);
/* device copies (domain box, NVAR comps): final state / adjoint of the state at
 * the window's first step (the initial state when first_step is 0) */
int    castro_adj_final_state(const castro_adj* adj, double* dst);
int    castro_adj_initial_adjoint(const castro_adj* adj, double* dst);
/* device time of the last forward (which=0) or backward (which=1) call, ms */
double castro_adj_time_ms(const castro_adj* adj, int which);
size_t castro_adj_device_bytes(const castro_adj* adj);

#ifdef __cplusplus
}
#endif
#endif
