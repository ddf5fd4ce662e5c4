/*
 * slg.h -- C ABI of the B200 (sm_100a) implementation of SuperLite's
 * per-timestep hot path: physical LTE opacity + Planck/Rosseland means, DDMC
 * leakage opacities and emission probabilities, the 1-D spherical IMC/DDMC
 * particle loop, and the flux and source tallies.
 *
 * Each entry point replaces one argument-less Fortran subroutine of the
 * reference (gururajw/superlite) that works on module arrays; the arrays it
 * reads and writes become explicit arguments, with the reference's
 * column-major layouts:  "(ng, ncell)" means group index fastest.
 *
 * Conventions
 *  - The caller owns every host array.  The library copies inputs to the GPU,
 *    runs, copies outputs back and keeps no host pointer after returning.
 *  - Return value 0 = success.  Transport errors reuse the reference's ierr
 *    codes (transport11: 1, 3, 4, 17; diffusion11: 100, 102) plus 1001 (the
 *    per-particle step guard); library errors are negative (SLG_ERR_*).
 *    slg_last_error() gives a message.  The library never exits the process.
 *  - Fortran logicals are passed as int32 0/1.
 *  - A context is bound to one device and one stream and is not re-entrant;
 *    calls on one context must come from one host thread at a time.
 *  - The grid is 1-D spherical without void cells: grd_icell(ix,1,1) = ix and
 *    ncell = nx.
 *  - Entry points named slg_dev_* take device pointers (and run on the
 *    context's stream without host synchronisation); the others take host
 *    pointers.
 */
#ifndef SLG_H
#define SLG_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SLG_OK 0
#define SLG_ERR_CUDA (-1)      /* a CUDA call failed (message in slg_last_error) */
#define SLG_ERR_ARG (-2)       /* invalid argument or shape */
#define SLG_ERR_STATE (-3)     /* required set-up call missing */
#define SLG_ERR_UNSORTED (-4)  /* bb line list not sorted by wl0 */
#define SLG_ERR_OOM (-5)       /* device allocation failed */
#define SLG_ERR_NOT_BUILT (-6) /* kernel variant not compiled in */
#define SLG_ERR_TOO_LARGE (-7) /* size beyond a documented limit */

/* Most groups a context or call accepts: per-cell group lists are int16, as
 * the reference's DDMC lump lists are (integer*2 glumps, diffusion11.f90:49,116). */
#define SLG_MAX_GROUPS 32767

typedef struct slg_ctx slg_ctx;

/* Line record, bbxsmod.f:27-34 (type bb_xs_data, 16 bytes). */
typedef struct slg_bbxs {
  float wl0;   /* line centre [Angstrom] */
  float gxs;   /* g * f * pi e^2 / (m_e c) */
  float chilw; /* lower level energy [cm^-1] */
  int16_t iz;  /* element */
  int16_t ii;  /* ion stage, 1 = neutral */
} slg_bbxs;

/* Particle record, particlemod.f90:7-11 (type packet, 64 bytes). */
typedef struct slg_packet {
  double x, y, z, mu, om, e, e0, wl;
} slg_packet;

/* ------------------------------------------------------------------ set-up */

/* Create a context on CUDA device `device` (its own stream).  NULL on failure. */
slg_ctx* slg_create(int device);
void slg_destroy(slg_ctx* ctx);
const char* slg_last_error(const slg_ctx* ctx);
/* Library version string (build date + compiled arch). */
const char* slg_version(void);

/* groupmod_init (groupmod.f:29-96): grp_wl(ng+1) in cm, increasing.  Also sets
 * grd_nep = nint(sqrt(ng)), grd_nepg = ceiling(ng/(nep+1)) (gridmod.f:121-122).
 * ng > SLG_MAX_GROUPS returns SLG_ERR_TOO_LARGE. */
int slg_set_groups(slg_ctx* ctx, int32_t ng, const double* grp_wl);

/* grid_setup + grid_volume (GRID/grid_setup.f:3-62, GRID/grid_volume.f:66-105):
 * grd_xarr(nx+1), grd_vxarr(nx+1), grd_vol(nx), grd_divv(nx). */
int slg_set_grid(slg_ctx* ctx, int32_t nx, const double* xarr, const double* vxarr,
                 const double* vol, const double* divv);

/* Many independent ejecta models in one context (no counterpart in the
 * reference, which runs one model per process).  Model m has nx[m] >= 2
 * shells and npart[m] particle slots.  xarr and vxarr hold each model's
 * nx[m]+1 shell edges, one model after the other; vol and divv each model's
 * nx[m] cells.  Every per-cell array of the other calls (temperatures, gas,
 * opacities, tallies ...) then runs over the sum of nx[m] cells in model
 * order, and the particle arrays over the sum of npart[m] slots in model order
 * (model m owns slots [npart[0] + ... + npart[m-1], + npart[m])).  Shell
 * neighbours never cross a model.  Per-model behaviour: sourceenergy
 * renormalises each model to L_bol, slg_models_sourcenumbers fills each
 * model's slots, interior_source writes each model's particles into its own
 * slots, fluxtally returns one row of flx_ng groups per model, and transport
 * (either precision) advances all models' particles in one persistent launch
 * (per-particle traces, slg_set_trace, are for one-model contexts).
 * Random numbers: model m draws under the key seed + m * SLG_MODEL_SEED_STRIDE
 * with slot numbers counted from the model's first slot, so each model
 * reproduces its own single-model run under that key. */
#define SLG_MODEL_SEED_STRIDE 0x9E3779B97F4A7C15ULL
int slg_set_models(slg_ctx* ctx, int32_t nmodel, const int32_t* nx, const int64_t* npart,
                   const double* xarr, const double* vxarr, const double* vol, const double* divv);

/* Permanent atomic data after bcast_permanent (mpimod_mpi.f:23-501):
 * ion_el(iz)%ni (nelem), the bb line list sorted by wl0 (read_bbxs_data.f:84),
 * bf_ph1(6,7,30,30), bf_ph2(7,30,30) (bfxsmod.f:14) and ff_gff(81,41)
 * (ffxsmod.f:18-20).  nstage = slots per element in the oc/ginv arrays
 * (1..64; nelem 1..30). */
int slg_set_atomic_data(slg_ctx* ctx, int32_t nelem, int32_t nstage, const int32_t* ion_ni,
                        int64_t nline, const slg_bbxs* bb_xs, const float* bf_ph1,
                        const float* bf_ph2, const double* ff_gff);

/* ------------------------------------------------------------------ equation of state */

/* Partition functions of ions_solve_eos (ionsmod.f:206-215) at temperature
 * temp (host computation): q(ii,iz) = sum_k glev(k,ii,iz) exp(-elev(k,ii,iz)/kT)
 * for stages 1..ni-1 and 1 for stage ni.  glev, elev (nlev, nstage, nelem) with
 * elev in erg, nlevel (nstage, nelem), q (nstage, nelem).  The reference
 * evaluates them once, at the temperature of the first cell of its first EOS
 * call, and keeps them. */
void slg_partition_functions(int32_t nelem, int32_t nstage, int32_t nlev, const int32_t* ni,
                             const int32_t* nlevel, const double* glev, const double* elev,
                             double temp, double* q);

/* Ion data of the equation of state (ionsmod.f ion_el after ions_read_data):
 * ni (nelem) stages including the bare ion, and (nstage, nelem) each: e the
 * ionisation energy of stage ii to ii+1 [erg], q the partition functions,
 * g1 the ground-level weights glev(1).  nelem <= 32, nstage <= 32. */
int slg_set_ions(slg_ctx* ctx, int32_t nelem, int32_t nstage, const int32_t* ni, const double* e,
                 const double* q, const double* g1);

/* ions_solve_eos (ionsmod.f:160-356) for every cell, then eos_update's ground
 * states (GAS/eos_update.f:37-45).  nelec (ncell) is the start value on entry
 * (the previous step's, as in the reference) and the converged electrons per
 * atom on return; acc is the convergence limit on |nelec/nelec_new - 1|
 * (reference 1e-8).  oc, ginv (ncell, noc, nelem) for stages 1..noc (0 and 1
 * beyond ni); iconv (ncell, optional) the iteration count (41: not converged,
 * -1: a cell where the reference stops).  natomfr is (0:nelem, ncell). */
int slg_saha_eos(slg_ctx* ctx, const double* temp, const double* natom, const double* vol,
                 const double* natomfr, double acc, double* nelec, int32_t noc, double* oc,
                 double* ginv, int32_t* iconv);

/* ------------------------------------------------------------------ opacity */

/* Gas state read by physical_opacity (gasmod.f), all per shell (ncell = nx). */
typedef struct slg_gas {
  const double* temp;    /* gas_temp (ncell) */
  const double* natom;   /* gas_natom (ncell) */
  const double* nelec;   /* gas_nelec (ncell), electrons per atom */
  const double* vol;     /* gas_vol (ncell) */
  const double* mass;    /* gas_mass (ncell) */
  const double* natomfr; /* gas_natomfr (0:nelem, ncell) */
  const double* oc;      /* ion_grndlev(iz,i)%oc(ii) as (ncell, nstage, nelem) */
  const double* ginv;    /* ion_grndlev(iz,i)%ginv(ii) as (ncell, nstage, nelem) */
} slg_gas;

typedef struct slg_opacity_flags {
  int32_t nobb, nobf, noff, nothmson; /* in_nobbopac, in_nobfopac, in_noffopac, in_nothmson */
  int32_t ngs;                        /* in_grp_ngs sub-groups per group (>= 1) */
  double opacmixrossel;               /* in_opacmixrossel */
} slg_opacity_flags;

/* physical_opacity (GAS/physical_opacity.f:3-357).  Outputs gas_sig (ncell),
 * gas_cap (ng, ncell) real*4, gas_emiss (ng, ncell) real*4 and optionally
 * cap64 (ncell, ng), the double opacity before sngl() (:267).  *sanity
 * (optional) receives the bitmask of the checks at :282-291. */
int slg_physical_opacity(slg_ctx* ctx, const slg_gas* gas, const slg_opacity_flags* flags,
                         double* gas_sig, float* gas_cap, float* gas_emiss, double* cap64,
                         int32_t* sanity);

/* analytic_opacity (GAS/analytic_opacity.f90:3-77).  kind: 1 grey, 2 mono, 3 line. */
int slg_analytic_opacity(slg_ctx* ctx, const double* temp, const double* rho, int32_t kind,
                         double capcoef, double captpwr, double caprpwr, double sigcoef,
                         double sigtpwr, double sigrpwr, double ldisp1, double ldisp2,
                         double* gas_sig, float* gas_cap);

/* opacity_planckmean + opacity_rossmean (GAS/opacity_planckmean.f:17-24,
 * GAS/opacity_rossmean.f:17-21): gas_capgrey, gas_capross (ncell). */
int slg_opacity_means(slg_ctx* ctx, const double* temp, const double* sig, const float* gas_cap,
                      double* capgrey, double* capross);

/* ------------------------------------------------------------------ grid coefficients */

/* leakage_opacity11 (GRID/leakage_opacity11.f90:3-174): grd_opaclump (11, ncell).
 * capemit (ng, ncell) may be NULL (LTE: treated as zero). */
int slg_leakage_opacity11(slg_ctx* ctx, const double* tempinv, const double* sig,
                          const float* cap, const float* capemit, double tauddmc,
                          double taulump, double* opaclump);

/* emission_probability (GRID/emission_probability.f90:3-67, LTE): grd_emitprob (nep, ncell). */
int slg_emission_probability(slg_ctx* ctx, const double* tempinv, const float* cap,
                             const double* capgrey, double* emitprob);

/* ------------------------------------------------------------------ transport */

/* Grid/opacity state read by particle_advance (gridmod.f, transportmod.f). */
typedef struct slg_transport_in {
  const double* tempinv;   /* grd_tempinv (ncell) */
  const double* sig;       /* grd_sig (ncell) */
  const double* capgrey;   /* grd_capgrey (ncell) */
  const double* emitprob;  /* grd_emitprob (nep, ncell) */
  const double* opaclump;  /* grd_opaclump (11, ncell) */
  const float* cap;        /* grd_cap (ng, ncell) */
  double tauddmc;          /* trn_tauddmc */
  double taulump;          /* trn_taulump */
  int32_t puretran, noampfact, errorfatal, thm_aniso, dogrdtally;
  int32_t precision;       /* 0: FP64 (reference arithmetic); 1: mixed FP32/FP64 */
  int64_t max_steps;       /* per-particle step guard; 0 = none */
} slg_transport_in;

/* Tallies written by particle_advance.  tally/eamp/methodswap (ncell),
 * jrad (ng, ncell) are overwritten (particle_advance.f90:65-72); the tot_*
 * fields accumulate into the caller's values (totalsmod.f). */
typedef struct slg_transport_out {
  double* tally;
  double* jrad;
  double* eamp;
  int32_t* methodswap;
  double tot_evelo, tot_eout, tot_sflux;
  int64_t npckt, nflux, nstepimc, nstepddmc, nmethodswap, nstepmax;
  int64_t ndist[11];       /* ndist(-3:7) */
  int64_t nposwarn;        /* ierr = -99 position warnings */
  int32_t ierr;            /* first fatal transport error (lowest particle index) */
  int32_t ierr_part;       /* its 1-based particle index */
} slg_transport_out;

/* particle_advance (particle_advance.f90:4-327) with transport11 / diffusion11
 * (TRANSPORT1/transport11.f90, TRANSPORT1/diffusion11.f90).  Random numbers:
 * one Philox4x32-10 stream per particle keyed by `seed` (replaces the
 * per-thread mzran streams of randommod.f).  prt (npart) and isvacant (npart,
 * logical as int32) are updated in place: dead particles become vacant,
 * escaped ones keep x = huge (:283-288). */
int slg_particle_advance(slg_ctx* ctx, const slg_transport_in* in, slg_packet* prt,
                         int32_t* isvacant, int64_t npart, uint64_t seed,
                         slg_transport_out* out);

/* Optional per-particle event trace of the next particle_advance call on this
 * context: an FNV-1a hash of (idist, itype, ic, ig, stat) after every event and
 * the step count, for parity tests.  Host arrays of npart entries; pass NULLs
 * to disable. */
int slg_set_trace(slg_ctx* ctx, uint64_t* trace_hash, int32_t* trace_nstep);

/* fluxtally (fluxtally.f:3-61) on flux grid flx_wl (flx_ng+1) with one polar
 * and one azimuthal bin (in_flx_ndim = ng,1,1): luminos, lumdev (flx_ng) and
 * lumnum (flx_ng); tallied slots become vacant. */
int slg_fluxtally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, int32_t* isvacant,
                  int32_t flx_ng, const double* flx_wl, double* luminos, double* lumdev,
                  int32_t* lumnum);

/* sourcetally (sourcetally.f:3-48): src_energy, src_number (ncell, ng). */
int slg_sourcetally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, const int32_t* isvacant,
                    double* src_energy, int32_t* src_number);

/* ------------------------------------------------------------------ sources */

/* sourceenergy (SOURCE/sourceenergy.f90:21-29): grd_emit (ncell) of the
 * surface-like thermal source, renormalised to L_bol; tot_sthermal optional.
 * Host arrays, host computation (O(ncell)). */
int slg_sourceenergy(slg_ctx* ctx, const double* radtemp, double L_bol, double* emit,
                     double* tot_sthermal);

/* sourcenumbers (SOURCE/sourcenumbers.f90:3-94, one rank, no surface source):
 * grd_nvol (ncell) for src_ns particles.  Returns src_nnew (>= 0) or a negative
 * error (vacancies < emitting cells, no particles, surplus > ncell). */
int64_t slg_sourcenumbers(slg_ctx* ctx, const double* emit, double srcepwr, int64_t src_ns,
                          int64_t nvacant, int32_t* nvol);
/* sourcenumbers for each model of slg_set_models: src_ns[m] particles and
 * nvacant[m] vacancies for model m; nvol over all cells.  Returns the total
 * src_nnew or a negative error. */
int64_t slg_models_sourcenumbers(slg_ctx* ctx, const double* emit, double srcepwr,
                                 const int64_t* src_ns, const int64_t* nvacant, int32_t* nvol);

/* vacancies + interior_source + source_transformdirection
 * (SOURCE/vacancies.f90, SOURCE/interior_source.f90:3-172,
 * SOURCE/source_transformdirection.f90:3-47): fills the first src_nnew vacant
 * slots of prt/isvacant with thermal source particles (lab-frame direction,
 * comoving energy and wavelength).  Random numbers: Philox4x32-10, one stream
 * per particle slot keyed by `seed` (stream 1).  *nnew receives src_nnew. */
int slg_interior_source(slg_ctx* ctx, const double* radtemp, const double* emit,
                        const int32_t* nvol, slg_packet* prt, int32_t* isvacant, int64_t npart,
                        uint64_t seed, int64_t* nnew);

/* ------------------------------------------------------------------ device-pointer forms */
/* Same semantics as above; every array argument is a device pointer, work is
 * queued on the context's stream, and the call returns after queueing (the
 * transport counters in *out are only valid after slg_sync()). */
int slg_dev_physical_opacity(slg_ctx* ctx, const slg_gas* gas, const slg_opacity_flags* flags,
                             double* gas_sig, float* gas_cap, float* gas_emiss, double* cap64);
int slg_dev_opacity_means(slg_ctx* ctx, const double* temp, const double* sig,
                          const float* gas_cap, double* capgrey, double* capross);
int slg_dev_analytic_opacity(slg_ctx* ctx, const double* temp, const double* rho, int32_t kind,
                             double capcoef, double captpwr, double caprpwr, double sigcoef,
                             double sigtpwr, double sigrpwr, double ldisp1, double ldisp2,
                             double* gas_sig, float* gas_cap);
int slg_dev_saha_eos(slg_ctx* ctx, const double* temp, const double* natom, const double* vol,
                     const double* natomfr, double acc, double* nelec, int32_t noc, double* oc,
                     double* ginv, int32_t* iconv);
int slg_dev_leakage_opacity11(slg_ctx* ctx, const double* tempinv, const double* sig,
                              const float* cap, const float* capemit, double tauddmc,
                              double taulump, double* opaclump);
int slg_dev_emission_probability(slg_ctx* ctx, const double* tempinv, const float* cap,
                                 const double* capgrey, double* emitprob);
int slg_dev_particle_advance(slg_ctx* ctx, const slg_transport_in* in, slg_packet* prt,
                             int32_t* isvacant, int64_t npart, uint64_t seed,
                             slg_transport_out* out);
int slg_dev_fluxtally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, int32_t* isvacant,
                      int32_t flx_ng, const double* flx_wl, double* luminos, double* lumdev,
                      int32_t* lumnum);
int slg_dev_sourcetally(slg_ctx* ctx, int64_t npart, const slg_packet* prt,
                        const int32_t* isvacant, double* src_energy, int32_t* src_number);
/* Transport autotuner (library addition): runs each compiled variant of the
 * particle-loop kernel of in->precision (register budget / resident blocks
 * per SM) on a copy of the first nsample particles (device pointers; inputs
 * are left unchanged), times it and keeps the fastest for this context and
 * precision.  *best (optional) receives the variant, ms (optional, 4
 * entries) the times. */
int slg_autotune_transport(slg_ctx* ctx, const slg_transport_in* in, const slg_packet* prt,
                           const int32_t* isvacant, int64_t npart, uint64_t seed,
                           int64_t nsample, int32_t* best, float* ms);
/* Select the transport kernel variant (0..3, register budget / resident
 * blocks, as slg_autotune_transport times them) of both precisions explicitly,
 * e.g. after timing each on full launches of the caller's own workload.  A new
 * context starts with FP64 variant 2 and mixed variant 3, the fastest on whole
 * steps of a large batched workload. */
int slg_set_transport_variant(slg_ctx* ctx, int32_t variant);
/* radtemp, prt and isvacant on the device; emit and nvol are host arrays. */
int slg_dev_interior_source(slg_ctx* ctx, const double* radtemp, const double* emit,
                            const int32_t* nvol, slg_packet* prt, int32_t* isvacant,
                            int64_t npart, uint64_t seed, int64_t* nnew);
/* ------------------------------------------------------------------ no device allocation */

/* Size limits of slg_particle_advance_static (see below).  Its group count is
 * also bounded by SLG_MAX_GROUPS, like every other entry point. */
#define SLG_STATIC_MAX_CELLGROUPS 131072 /* ncell * ng */
#define SLG_STATIC_MAX_CELLS 4096

/* Grid and group arrays on the device (grd_xarr, grd_vxarr (nx+1), grd_divv
 * (nx), grp_wl, grp_wlinv (ng+1)), for the entry point below. */
typedef struct slg_grid_dev {
  int32_t nx, ng;
  const double* xarr;
  const double* vxarr;
  const double* divv;
  const double* wl;
  const double* wlinv;
} slg_grid_dev;

/* particle_advance for callers that cannot allocate device memory (no
 * counterpart in the reference: an addition of this library).  Same semantics
 * as slg_dev_particle_advance, but needs no context and calls no allocator:
 * every input and output is a caller-owned device pointer, and the per-cell
 * tables and counters live in one fixed 6.5 MiB __device__ array that every GPU
 * loading the library holds until exit.  Grids beyond SLG_STATIC_MAX_CELLS
 * shells or SLG_STATIC_MAX_CELLGROUPS (shells x groups) return
 * SLG_ERR_TOO_LARGE.  Runs on `stream` (a cudaStream_t, NULL = default) on the
 * current device and returns after the stream has finished it.  The first
 * call on a device looks up the array's device address; make it before any
 * stream capture.  The address is kept per device for the life of the
 * process, so do not call this entry point again after cudaDeviceReset (which
 * unloads the array).  All calls share the array: calls that overlap on the
 * GPU race, so serialise them. */
int slg_particle_advance_static(const slg_grid_dev* grid, const slg_transport_in* in,
                                slg_packet* prt, int32_t* isvacant, int64_t npart,
                                uint64_t seed, slg_transport_out* out, void* stream);

/* ------------------------------------------------------------------ differentiable opacity */
/* The opacity build as a differentiable function of shell temperature,
 * density and mass fractions, with a hand-written reverse mode (no
 * counterpart in the reference).  Needs groups, grid (one model), atomic data,
 * ion data for the same nelem elements and their masses.  Device pointers. */

/* Element masses [amu] of elements 1..nelem (elemdatamod elem_data%m). */
int slg_set_element_masses(slg_ctx* ctx, int32_t nelem, const double* mass_amu);

/* Forward: massfr2natomfr (GAS/gas_setup.f:101-160; massfr (nelem, ncell),
 * renormalised per shell), the equation of state (slg_saha_eos at accuracy
 * acc; nelec in/out), physical_opacity with ngs = 1 and the FP64 opacity
 * returned in cap (ng, ncell) (gas_cap's layout before sngl), sig (ncell),
 * opacity_planckmean / rossmean and leakage_opacity11 computed on that FP64
 * opacity: capgrey, capross (ncell), opaclump (11, ncell). */
int slg_dev_opacity_grad_forward(slg_ctx* ctx, const double* temp, const double* rho,
                                 const double* massfr, double acc, double tauddmc,
                                 double taulump, double* nelec, double* cap, double* sig,
                                 double* capgrey, double* capross, double* opaclump);

/* Reverse mode of slg_dev_opacity_grad_forward: given its inputs, its nelec
 * and outputs, and dL/d(cap, sig, capgrey, capross, opaclump) (NULL = zero;
 * opaclump rows 1, 2, 7, 8, 11 carry gradients), writes dL/dtemp, dL/drho
 * (ncell) and dL/dmassfr (nelem, ncell).  The equation of state enters
 * through its implicit derivative at the returned solution, so pass acc near
 * machine precision (1e-14) when the gradient must match finite differences. */
int slg_dev_opacity_grad_backward(slg_ctx* ctx, const double* temp, const double* rho,
                                  const double* massfr, double acc, double tauddmc,
                                  double taulump, const double* nelec, const double* cap,
                                  const double* sig, const double* capgrey,
                                  const double* capross, const double* opaclump,
                                  const double* gcap, const double* gsig, const double* gcapgrey,
                                  const double* gcapross, const double* gopaclump, double* gtemp,
                                  double* grho, double* gmassfr);

/* ------------------------------------------------------------------ CUDA graphs */
/* Capture the work that slg_dev_* calls queue on the context's stream
 * between slg_graph_begin and slg_graph_end into one executable CUDA graph
 * held by the context (no counterpart in the reference).  Make one
 * uncaptured pass of the same calls first: a call that needs a new device
 * buffer, an upload of changed host data (interior_source re-uploads its
 * set-up only when emit/nvol change) or a host wait makes slg_graph_end
 * fail.  slg_graph_launch replays the graph nlaunch times.  Replay r, counted
 * from 0 after slg_graph_end, draws every random number of the captured
 * transport and source calls from the Philox counter word
 * 3 = stream | r << 2, so replay 0 equals the same calls made directly and
 * later replays draw fresh numbers.  Transport counters of replays are read
 * with slg_transport_totals. */
int slg_graph_begin(slg_ctx* ctx);
int slg_graph_end(slg_ctx* ctx);
int slg_graph_launch(slg_ctx* ctx, int32_t nlaunch);
/* Counters of every particle_advance (direct or replayed) since the context
 * was made or last reset, summed (nstepmax: maximum; ierr/ierr_part: the
 * lowest error key), written to the scalar fields of *out (tot_* are set, not
 * added); arrays of *out are not touched.  Waits for the stream; reset != 0
 * zeroes the sums.  Returns the first transport error code (0 if none). */
int slg_transport_totals(slg_ctx* ctx, slg_transport_out* out, int32_t reset);

/* Wait for the context's stream; returns a pending error if any. */
int slg_sync(slg_ctx* ctx);
/* The context's cudaStream_t, as an opaque handle. */
void* slg_stream(slg_ctx* ctx);

/* ------------------------------------------------------------------ pipe throughput */
/* Throughput microbenchmark of one pipe of device `device` (no counterpart in
 * the reference; the denominators of the kernels' rooflines): which = 0 FP64
 * fused multiply-add (flop/s, 2 per FMA), 1 FP64 exp (evaluations/s), 2 FP32
 * fused multiply-add (flop/s), 3 32-bit integer multiply-add (operations/s).
 * One launch of 8 blocks x 256 threads per SM, `iters` rounds of independent
 * chains per thread, timed with CUDA events after one warm-up launch; *ms
 * (optional) receives the launch time.  Allocates and frees its own buffer. */
int slg_pipe_throughput(int device, int which, int iters, double* ops_per_s, float* ms);

/* y[k] = the opacity kernels' FP64 exp (Tang's table-driven method) of x[k]
 * on device `device`, k < n (host arrays; no counterpart in the reference: an
 * accuracy check of that exp against a host libm).  Synchronous. */
int slg_exp_eval(int device, int64_t n, const double* x, double* y);

#ifdef __cplusplus
}
#endif
#endif
