/*
 * castro_oracle.h -- CPU oracle for mini-Castro's CTU hydro advance.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (mini-castro_b200/) links,
 * loads or calls this code; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py use it, as the checker.
 *
 * PARITY UNPINNED: the reference (Fortran + AMReX) cannot be compiled in this
 * image (no Fortran compiler, empty AMReX submodule) and ships no golden
 * vectors, so this restatement is pinned only by internal consistency checks
 * (EOS node exactness and round trips, conservation, symmetry, blast growth).
 *
 * Every routine restates one reference routine; the file:line it follows is
 * cited beside its definition in castro_oracle.c.  Array arguments use the
 * reference's BL_FORT_FAB_ARG_3D convention: (pointer, lo[3], hi[3]) with
 * Fortran order (i fastest, component slowest); lo/hi are inclusive.
 * Component indices are 0-based here (the Fortran ones are 1-based).
 */
#ifndef CASTRO_ORACLE_H
#define CASTRO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_SPEC 13

/* eos_t, Source/eos.F90:18-58 */
typedef struct {
    double rho, T, p, e, h, s, abar, zbar;
    double dpdT, dpdr, dedT, dedr, dhdT, dhdr, dsdT, dsdr, dpde, dpdr_e;
    double cv, cp, xne, xnp, eta, pele, ppos, mu, mu_e, y_e, gam1, cs;
    double dpdA, dpdZ, dedA, dedZ;
} oracle_eos_t;

/* eos input modes, Source/eos.F90:11-13 */
#define ORACLE_EOS_INPUT_RT 1
#define ORACLE_EOS_INPUT_RE 2
#define ORACLE_EOS_INPUT_RP 3

/* Sedov problem description (Source/Prob.F90:11-15 plus the knobs the
 * benchmark configurations need). */
typedef struct {
    int    ambient_from_T;   /* 0: ambient e from EOS(rho,p) as Prob.F90; 1: from EOS(rho,T) */
    double dens_ambient;     /* g/cc */
    double p_ambient;        /* erg/cc, used when ambient_from_T == 0 */
    double T_ambient;        /* K, used when ambient_from_T == 1 */
    double exp_energy;       /* erg */
    double r_init;           /* cm */
    int    nsub;             /* subgrid zones per dimension */
    double X[ORACLE_MAX_SPEC];     /* initial mass fractions */
    double T_init;           /* value stored in UTEMP at init (Prob.F90:115 uses 1e9) */
    /* optional density perturbation rho = dens_ambient*(1 + amp*pert(i,j,k)),
     * pert indexed over the domain box pert_lo..pert_hi (Fortran order) */
    const double* pert;
    int    pert_lo[3], pert_hi[3];
    double pert_amp;
} oracle_prob_t;

int  oracle_network_init(int nspec, const double* aion, const double* zion);
int  oracle_nspec(void);
int  oracle_eos_init(const char* path);
void oracle_eos_finalize(void);
void oracle_eos(int input, oracle_eos_t* state);
void oracle_set_problem(const oracle_prob_t* prob);
/* the interface pressure in the normal momentum flux (off by default, as in the reference) */
void oracle_set_momentum_flux_pressure(int on);
/* Coulomb corrections in the EOS (off by default, as in the reference's eos.F90) */
void oracle_set_coulomb_corrections(int on);

/* Source/Castro_F.H entry points, same argument order and meaning. */
void oracle_ctoprim(const int* lo, const int* hi,
                    const double* u, const int* u_lo, const int* u_hi,
                    double* q, const int* q_lo, const int* q_hi,
                    double* qaux, const int* qa_lo, const int* qa_hi);
void oracle_enforce_minimum_density(const int* lo, const int* hi, double* u, const int* u_lo, const int* u_hi);
void oracle_normalize_species(const int* lo, const int* hi, double* u, const int* u_lo, const int* u_hi);
void oracle_reset_internal_e(const int* lo, const int* hi, double* u, const int* u_lo, const int* u_hi);
void oracle_compute_temp(const int* lo, const int* hi, double* u, const int* u_lo, const int* u_hi);
void oracle_estdt(const int* lo, const int* hi, const double* u, const int* u_lo, const int* u_hi,
                  const double* dx, double* dt);
void oracle_store_flux(const int* lo, const int* hi,
                       double* fo, const int* fo_lo, const int* fo_hi,
                       const double* fi, const int* fi_lo, const int* fi_hi,
                       const double* area, const int* a_lo, const int* a_hi, double dt);
void oracle_fill_hydro_source(const int* lo, const int* hi,
                              const double* u, const int* u_lo, const int* u_hi,
                              const double* q, const int* q_lo, const int* q_hi,
                              double* src, const int* s_lo, const int* s_hi,
                              const double* f1, const int* f1_lo, const int* f1_hi,
                              const double* f2, const int* f2_lo, const int* f2_hi,
                              const double* f3, const int* f3_lo, const int* f3_hi,
                              const double* qx, const int* qx_lo, const int* qx_hi,
                              const double* qy, const int* qy_lo, const int* qy_hi,
                              const double* qz, const int* qz_lo, const int* qz_hi,
                              const double* a1, const int* a1_lo, const int* a1_hi,
                              const double* a2, const int* a2_lo, const int* a2_hi,
                              const double* a3, const int* a3_lo, const int* a3_hi,
                              const double* vol, const int* v_lo, const int* v_hi,
                              const double* dx, double dt);
void oracle_normalize_species_fluxes(const int* lo, const int* hi, double* f, const int* f_lo, const int* f_hi);
void oracle_apply_av(const int* lo, const int* hi, int idir, const double* dx,
                     const double* div, const int* d_lo, const int* d_hi,
                     const double* u, const int* u_lo, const int* u_hi,
                     double* f, const int* f_lo, const int* f_hi);
void oracle_trans1(const int* lo, const int* hi, int idir1, int idir2,
                   const double* q2m, const int* q2m_lo, const int* q2m_hi,
                   double* q2mo, const int* q2mo_lo, const int* q2mo_hi,
                   const double* q2p, const int* q2p_lo, const int* q2p_hi,
                   double* q2po, const int* q2po_lo, const int* q2po_hi,
                   const double* qaux, const int* qa_lo, const int* qa_hi,
                   const double* f1, const int* f1_lo, const int* f1_hi,
                   const double* q1, const int* q1_lo, const int* q1_hi,
                   double cdtdx);
void oracle_trans2(const int* lo, const int* hi, int idir1, int idir2, int idir3,
                   const double* qm, const int* qm_lo, const int* qm_hi,
                   double* qmo, const int* qmo_lo, const int* qmo_hi,
                   const double* qp, const int* qp_lo, const int* qp_hi,
                   double* qpo, const int* qpo_lo, const int* qpo_hi,
                   const double* qaux, const int* qa_lo, const int* qa_hi,
                   const double* f2, const int* f2_lo, const int* f2_hi,
                   const double* f3, const int* f3_lo, const int* f3_hi,
                   const double* q2, const int* q2_lo, const int* q2_hi,
                   const double* q3, const int* q3_lo, const int* q3_hi,
                   double hdtdx, double cdtdy, double cdtdz);
void oracle_compute_flux(const int* lo, const int* hi,
                         const double* ql, const int* ql_lo, const int* ql_hi,
                         const double* qr, const int* qr_lo, const int* qr_hi,
                         double* flx, const int* fx_lo, const int* fx_hi,
                         double* qint, const int* qi_lo, const int* qi_hi,
                         double* qe, const int* qe_lo, const int* qe_hi,
                         const double* qaux, const int* qa_lo, const int* qa_hi,
                         int idir);
void oracle_divu(const int* lo, const int* hi,
                 const double* q, const int* q_lo, const int* q_hi,
                 const double* dx, double* div, const int* d_lo, const int* d_hi);
void oracle_trace_ppm(const int* lo, const int* hi, const int* vlo, const int* vhi, int idir,
                      const double* q, const int* q_lo, const int* q_hi,
                      const double* qaux, const int* qa_lo, const int* qa_hi,
                      double* qm, const int* qm_lo, const int* qm_hi,
                      double* qp, const int* qp_lo, const int* qp_hi,
                      const int* domlo, const int* domhi, const double* dx, double dt);
void oracle_initdata(const int* lo, const int* hi, double* u, const int* u_lo, const int* u_hi,
                     const double* dx, const double* problo, const double* probhi);
void oracle_denerror(const int* lo, const int* hi,
                     signed char* tag, const int* t_lo, const int* t_hi,
                     const double* den, const int* d_lo, const int* d_hi,
                     signed char tagval, signed char clearval);
void oracle_calculate_blast_radius(const int* lo, const int* hi,
                                   const double* u, const int* u_lo, const int* u_hi,
                                   const double* dx, const double* problo, const double* probhi,
                                   double* blast_mass, double* blast_radius, double max_density);

/* Castro::construct_hydro_source for one tile bx of one box
 * (Source/Castro_hydro.cpp:31-395): Sborder on grow(box,4) in, source on the
 * tile (accumulated, caller zeroes), optional fluxes_out[3] (face FABs of the
 * box, may be NULL). */
void oracle_construct_hydro_source_tile(const int* bx_lo, const int* bx_hi,
                                        const double* sb, const int* sb_lo, const int* sb_hi,
                                        double* src, const int* s_lo, const int* s_hi,
                                        const int* domlo, const int* domhi,
                                        const double* dx, double dt);

/* ---- single-level driver (Castro::advance and friends) ---- */
typedef struct oracle_level oracle_level;

/* bc: 0 = periodic (the reference's INT_DIR, Source/Castro_setup.cpp:58-63),
 *     1 = outflow (zero-gradient copy of the nearest valid zone). */
oracle_level* oracle_level_create(int nbox, const int* box_lo, const int* box_hi,
                                  const int* dom_lo, const int* dom_hi,
                                  const double* problo, const double* probhi, int bc);
void    oracle_level_destroy(oracle_level* lev);
double* oracle_level_state(oracle_level* lev, int ibox);
int     oracle_level_nbox(const oracle_level* lev);
void    oracle_level_set_threads(oracle_level* lev, int nthreads);
void    oracle_level_init_data(oracle_level* lev);
double  oracle_level_est_time_step(oracle_level* lev);
void    oracle_level_clean_state(oracle_level* lev);
void    oracle_level_advance(oracle_level* lev, double dt);
/* Amr::coarseTimeStep: dt choice (computeInitialDt on the first step,
 * computeNewDt afterwards), advance, post_timestep.  Returns the dt used. */
double  oracle_level_coarse_step(oracle_level* lev, double stop_time);
double  oracle_level_time(const oracle_level* lev);
double  oracle_level_dt(const oracle_level* lev);
int     oracle_level_steps(const oracle_level* lev);
/* Castro::post_timestep diagnostic (Source/Castro.cpp:371-424): returns the
 * blast radius in cm; blast_mass is written when non-NULL. */
double  oracle_level_blast_radius(oracle_level* lev, double* blast_mass);

#ifdef __cplusplus
}
#endif
#endif
