/*
 * superlite_oracle.h -- CPU restatement of SuperLite's per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * product in superlite_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * path never links, loads or calls anything in oracle/.
 *
 * Every function restates one Fortran routine of the reference (gururajw/superlite)
 * and cites it by file:line.  Restatement rules:
 *   - Fortran evaluation order is kept (left-to-right products, no FMA
 *     contraction: built with -ffp-contract=off);
 *   - real*4 fields are promoted to double exactly where Fortran mixed-mode
 *     arithmetic promotes them (e.g. real*4**2 is squared in single precision
 *     inside bfxs);
 *   - sngl() is a round-to-nearest double->float conversion;
 *   - indices are 1-based in the comments, 0-based in memory;
 *   - arrays are Fortran column-major: (ng,ncell) means group fastest.
 *
 * Parity with the reference is pinned by analytic known-answer tests
 * (tests/test_oracle_kats.py): the reference ships no golden vectors and
 * cannot be compiled in this environment (no Fortran compiler).
 */
#ifndef SUPERLITE_ORACLE_H
#define SUPERLITE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* bb line record, bbxsmod.f:27-34 (16 bytes). */
typedef struct orc_bbxs {
  float wl0;    /* line centre [Angstrom] */
  float gxs;    /* g * f * pi e^2/(m_e c) */
  float chilw;  /* lower level energy [cm^-1] */
  int16_t iz;   /* element (1..30) */
  int16_t ii;   /* ion stage (1 = neutral) */
} orc_bbxs;

/* ---------------- groupmod.f Planck integrals ---------------- */
double orc_specint0(double tempinv, const double* wlinv, int ig);
double orc_dopspeccalc(double tempinv, const double* wlinv, int ig);
/* specintv(tempinv,n,ss,offset,mode) groupmod.f:146-272; offset is 1-based. */
void orc_specintv(double tempinv, const double* wlinv, int ng, int n, int offset,
                  int mode, double* ss);
void orc_spectintv(double tempinv, const double* wlinv, int ng, int n, int offset,
                   int mode, double* ss);
double orc_planck(double wl, double temp);
int orc_binsrch(double x, const double* arr, int n, int widerange);

/* ---------------- LTE equation of state ---------------- */
/* Ion data of ions_read_data (ionsmod.f:652-829) for nelem elements, stage
 * slots per element nstage (>= every ni): ni (nelem) stages including the bare
 * ion; e (nstage, nelem) ionisation energy of stage ii to ii+1 [erg]; q
 * (nstage, nelem) partition functions; g1 (nstage, nelem) ground-level weights. */
typedef struct orc_ion {
  int32_t nelem, nstage;
  const int32_t* ni;
  const double* e;
  const double* q;
  const double* g1;
} orc_ion;
/* Partition functions as ions_solve_eos evaluates them (ionsmod.f:206-215) at
 * one temperature: q = sum_k glev exp(-elev/(kb temp)) for stages 1..ni-1,
 * 1 for stage ni.  glev, elev (nlev, nstage, nelem), nlevel (nstage, nelem). */
void orc_partition(int nelem, int nstage, int nlev, const int32_t* ni, const int32_t* nlevel,
                   const double* glev, const double* elev, double temp, double* q);
/* ions_solve_eos (ionsmod.f:160-356) and eos_update (GAS/eos_update.f:20-45)
 * for every cell: nelec (ncell) in/out, accuracy acc (reference 1e-8), oc and
 * ginv (ncell, noc, nelem) for stages 1..noc, iconv (ncell, optional) the
 * iteration count.  Returns 0, or -(cell+1) where the reference stops. */
int orc_saha_eos(const orc_ion* ion, int ncell, const double* temp, const double* natom, const double* vol,
                 const double* natomfr, double acc, double* nelec, int32_t noc, double* oc, double* ginv,
                 int32_t* iconv);

/* ---------------- opacity ---------------- */
double orc_bfxs(const float* bf_ph1, const float* bf_ph2, int nz, int ne, double e);

typedef struct orc_opac_in {
  int32_t ncell, ng, ngs, nelem, nstage;
  const double* grp_wl;       /* (ng+1) [cm] */
  const double* temp;         /* (ncell) */
  const double* natom;        /* (ncell) */
  const double* nelec;        /* (ncell) */
  const double* vol;          /* (ncell) */
  const double* mass;         /* (ncell) */
  const double* natomfr;      /* (0:nelem, ncell) */
  const int32_t* ion_ni;      /* (nelem) ion_el(iz)%ni */
  const double* oc;           /* (ncell, nstage, nelem) ion_grndlev%oc */
  const double* ginv;         /* (ncell, nstage, nelem) ion_grndlev%ginv */
  int64_t nline;
  const orc_bbxs* bb;         /* (nline), sorted by wl0 */
  const float* bf_ph1;        /* (6,7,30,30) */
  const float* bf_ph2;        /* (7,30,30) */
  const double* ff_gff;       /* (81,41) */
  int32_t nobb, nobf, noff, nothmson;
  double opacmixrossel;
} orc_opac_in;

/* physical_opacity, GAS/physical_opacity.f:3-357.
 * cap64 (ncell, ng) optional: the collapsed double opacity before sngl().
 * Returns the sanity-check bitmask of :282-291 (bit 1 zero, 2 negative, 4 NaN, 8 inf). */
int orc_physical_opacity(const orc_opac_in* in, double* gas_sig, float* gas_cap,
                         float* gas_emiss, double* cap64);

/* analytic_opacity, GAS/analytic_opacity.f90:3-77.  kind: 1 grey, 2 mono, 3 line. */
void orc_analytic_opacity(int ncell, int ng, const double* wlinv, const double* temp,
                          const double* rho, int kind, double capcoef, double captpwr,
                          double caprpwr, double sigcoef, double sigtpwr, double sigrpwr,
                          double ldisp1, double ldisp2, double* gas_sig, float* gas_cap);

void orc_opacity_planckmean(int ncell, int ng, const double* wlinv, const double* temp,
                            const float* gas_cap, double* capgrey);
void orc_opacity_rossmean(int ncell, int ng, const double* wlinv, const double* temp,
                          const double* sig, const float* gas_cap, double* capross);

/* ---------------- grid coefficients ---------------- */
void orc_leakage_opacity11(int nx, int ng, const double* xarr, const double* vol,
                           const double* divv, const double* tempinv, const double* sig,
                           const float* cap, const float* capemit, const double* wlinv,
                           double tauddmc, double taulump, double* opaclump);
void orc_emission_probability(int nx, int ng, int nep, int nepg, const double* tempinv,
                              const float* cap, const double* capgrey, const double* wlinv,
                              double* emitprob);
int orc_emitgroup(double r, int ic, int ng, int nep, int nepg, const double* tempinv,
                  const float* cap, const double* capgrey, const double* emitprob,
                  const double* wlinv);

/* ---------------- random numbers ---------------- */
/* mzran state, randommod.f:12-14 */
typedef struct orc_rnd { int32_t part[4]; } orc_rnd;
void orc_rnd_init(int n, int ioffset, orc_rnd* states);
double orc_rnd_r(orc_rnd* s);
/* Philox4x32-10 per-particle stream shared with the CUDA kernels. */
double orc_philox_draw(uint64_t seed, uint64_t pid, uint32_t stream, uint32_t k);

/* ---------------- transport ---------------- */
typedef struct orc_packet { double x, y, z, mu, om, e, e0, wl; } orc_packet;

typedef struct orc_trn_in {
  int32_t nx, ng, nep, nepg;
  const double* xarr;       /* (nx+1) */
  const double* vxarr;      /* (nx+1) */
  const double* divv;       /* (nx) */
  const double* wl;         /* (ng+1) */
  const double* wlinv;      /* (ng+1) */
  const double* tempinv;    /* (nx) */
  const double* sig;        /* (nx) */
  const double* capgrey;    /* (nx) */
  const double* emitprob;   /* (nep, nx) */
  const double* opaclump;   /* (11, nx) */
  const float* cap;         /* (ng, nx) */
  double tauddmc, taulump;
  int32_t puretran, noampfact, errorfatal, thm_aniso, dogrdtally;
  int64_t max_steps;        /* per-particle step guard (library addition) */
} orc_trn_in;

typedef struct orc_trn_out {
  double* tally;            /* (nx) grd_tally */
  double* jrad;             /* (ng, nx) */
  double* eamp;             /* (nx) */
  int32_t* methodswap;      /* (nx) */
  double tot_evelo, tot_eout, tot_sflux;   /* accumulated (inout) */
  int64_t npckt, nflux, nstepimc, nstepddmc, nmethodswap, nstepmax;
  int64_t ndist[11];        /* ndist(-3:7) */
  int64_t nposwarn;         /* ierr=-99 warnings */
  int32_t ierr;             /* first fatal transport error (0 = none) */
  int32_t ierr_part;        /* 1-based particle index of that error */
} orc_trn_out;

/* particle_advance, particle_advance.f90:4-327.
 * rngmode 0: faithful mzran, one stream per OpenMP thread, schedule(static,1);
 *            rnd_states (nthreads) is read and written back.
 * rngmode 1: Philox stream per particle (seed, pid = ipart-1, stream 0).
 * trace_hash/trace_nstep (optional, npart): per-particle event-sequence hash. */
int orc_particle_advance(const orc_trn_in* in, orc_packet* prt, int32_t* isvacant,
                         int64_t npart, int rngmode, uint64_t seed, int nthreads,
                         orc_rnd* rnd_states, orc_trn_out* out, uint64_t* trace_hash,
                         int32_t* trace_nstep);

/* fluxtally.f:3-61 (flx_nmu = flx_nom = 1 grid: mu in [-1,1], om in [0,2pi]). */
void orc_fluxtally(int64_t npart, const orc_packet* prt, int32_t* isvacant, int flx_ng,
                   const double* flx_wl, double* luminos, double* lumdev, int32_t* lumnum);
/* sourcetally.f:3-48; src_energy (ncell, ng) cell fastest. */
int orc_sourcetally(int64_t npart, const orc_packet* prt, const int32_t* isvacant, int nx,
                    int ng, const double* xarr, const double* wl, double* src_energy,
                    int32_t* src_number);

/* ---------------- sources (input generation) ---------------- */
void orc_sourceenergy(int nx, const double* xarr, const double* radtemp, double L_bol,
                      double* emit, double* tot_sthermal);
/* sourcenumbers.f90 for one rank, no surface source: returns src_nnew. */
int64_t orc_sourcenumbers(int nx, const double* emit, double srcepwr, int64_t src_ns,
                          int64_t nvacant, int32_t* nvol);
/* vacancies + interior_source + source_transformdirection.  rngmode 0: the
 * reference's single mzran stream `state`; 1: one Philox stream per particle
 * (seed, pid = slot index, stream 1), as the GPU source kernel draws. */
int orc_interior_source(int nx, int ng, const double* xarr, const double* vxarr,
                        const double* wlinv, const double* radtemp, const double* emit,
                        double srcepwr, const int32_t* nvol, int64_t npart,
                        orc_packet* prt, int32_t* isvacant, orc_rnd* state, int rngmode,
                        uint64_t seed);

#ifdef __cplusplus
}
#endif
#endif
