// fb_dev.cuh -- device-side data structures of libfargo_b200.so (internal).
//
// Memory layout in HBM: every 2-D field is one array of (nr+1)*ns doubles in
// the reference's ring-major order l = j + i*ns (src/LowTasks.c:97-112), so
// a ring is a contiguous, 8-byte aligned run of ns doubles and a warp reading
// 32 consecutive azimuths issues fully coalesced 256-byte transactions.
// Ring nr exists for the outer radial-velocity interface.  All scratch
// fields are zeroed once at creation; rings that the reference never writes
// in a scratch field therefore read as zero here too, which the step relies
// on (e.g. VradInt ring 0 and ring nr, src/SourceEuler.c:866 loops 1..nr-1).
#pragma once
#include <cuda_runtime.h>
#include "fb_internal.h"

// Device-resident control block: the scalar state of AlgoGas
// (src/SourceEuler.c:333-460), advanced by a one-thread kernel so that the
// whole substep stays on the device.
struct fb_ctl {
  double DT, dtemp, dt, dthydro, dtnbody;
  double physical_time, physical_time_initial, omega_frame;
  double mindt, maxdt, lost_mass;
  double disk_acc_x, disk_acc_y, disk_acc_alt_x, disk_acc_alt_y;
  double ind_x, ind_y;                       // IndirectTerm (Pframeforce.c:25)
  double bary_x[3], bary_y[3];               // stardiscbarycenter_{x,y}
  double mdisc;
  int substeps, done, status, nonfinite;
  // DetectCrash (SourceEuler.c:51-69) as AlgoGas uses it (:545-566): the
  // CFL kernel's CTAs raise the flags for the state at the start of the
  // substep, the controller consumes them.  Only the energy test decides a
  // crash there (its result overwrites the density test's, :546-548).
  int neg_dens_flag, neg_energy_flag;
  int crashes;            // AlreadyCrashed: crashed substeps since creation
  int crash_substeps;     // crashed substeps of this DT
  int neg_dens_substeps;  // substeps of this DT that began with a negative density
  int crash_snap_now;     // this substep's starting state is the first crash's
  int crash_snapped;      // the first crash's state is held (fb_download_crash)
  double crash_time;      // timeCRASH (SourceEuler.c:551)
  int np;
  unsigned int cfl_done;                     // CTAs of the CFL kernel finished this substep
  double pm[FB_MAX_PLANETS], px[FB_MAX_PLANETS], py[FB_MAX_PLANETS];
  double pvx[FB_MAX_PLANETS], pvy[FB_MAX_PLANETS], pacc[FB_MAX_PLANETS];
  double pinit[FB_MAX_PLANETS], pfinal[FB_MAX_PLANETS];
  int pfeelothers[FB_MAX_PLANETS];
  // planets as seen by FillForcesArrays in the current substep
  double pot_m[FB_MAX_PLANETS], pot_x[FB_MAX_PLANETS], pot_y[FB_MAX_PLANETS];
  double pot_smooth2[FB_MAX_PLANETS], pot_invd3[FB_MAX_PLANETS];
  double t_sub;  // PhysicalTime at the start of the substep (FillForcesArrays' time)
  double domega; // corotating frame: this substep's change of OmegaFrame (CorrectVtheta)
  // implicit radiative diffusion (SubStep0, SourceEuler.c:749-760): the
  // relaxation parameter omegaSOR and the previous solve's iteration count
  // niterbuf, both carried from solve to solve; sor_iters = the last solve's
  double sor_omega;
  int sor_niterbuf, sor_iters;
};
#define FB_SOR_MAXITS 100000  // MAXITS of SourceEuler.c:20
#define FB_SOR_OMEGA0 1.97    // omegaSOR's initial value (SourceEuler.c:47)
#define FB_SOR_EPS 1e-4       // epsilonSOR (SourceEuler.c:48)

// Turbulent potential (ApplyLSAOnPotential, src/turb.c:13-135): the modes'
// parameters, the drand48 stream they are drawn from, and per substep each
// mode's time factor sin(pi ttilde / deltat) and the cosine and sine of its
// phase phic + (omegac - OmegaFrame) ttilde.  act[0 .. nact) lists the modes
// that add to the potential (all of them unless HIGHMCUTOFF, then m <= 6),
// in mode order.
struct fb_lsa {
  unsigned long long x;
  int nact, status;
  int m[FB_LSA_MAX_MODES], redraw[FB_LSA_MAX_MODES], act[FB_LSA_MAX_MODES];
  double rc[FB_LSA_MAX_MODES], phic[FB_LSA_MAX_MODES], xi[FB_LSA_MAX_MODES];
  double omegac[FB_LSA_MAX_MODES], sigma[FB_LSA_MAX_MODES], deltat[FB_LSA_MAX_MODES];
  double t0[FB_LSA_MAX_MODES], tf[FB_LSA_MAX_MODES];
  double s[FB_LSA_MAX_MODES], cp[FB_LSA_MAX_MODES], sp[FB_LSA_MAX_MODES];
};

// Everything a kernel needs, passed by value (well under the 32 KB limit).
struct KP {
  int nr, ns;
  size_t nf;
  // state
  double *rho, *vr, *vt, *e;
  // derived / scratch fields
  double *cs, *pres, *pot;
  double *vri, *vti;
  double *divv, *trr, *tpp, *trp, *vischeat;
  double *q[6];        // transport: RadMomP, RadMomM, ThetaMomP, ThetaMomM, Energy, Rho
  double *rho_t;       // density after transport, before floors
  // tile variant of the azimuthal pass: RadMomP and RadMomM after the radial
  // pass and a copy of vtheta (three fields), and the ring means of vtheta
  // (nr); vt_copy is azt_buf[2] in the radial pass feeding the tile variant,
  // else NULL
  double *azt_buf[3], *azt_vmed, *vt_copy;
  double *crash_snap;  // 4 x nr*ns: density, vrad, vtheta, energy of the first crash
  double *lost0;       // ns: ring-0 radial mass fluxes of the last substep
  double *sg_accr, *sg_acct;  // SG accelerations (nf)
  // per-ring tables (nr or nr+1 entries)
  const double *rinf, *rsup, *rmed, *surf, *invrmed, *invsurf, *invdiffrsup, *invrinf, *invdiffrmed;
  const double *cosaz, *sinaz;
  const double *cs_ring;   // isothermal sound speed per ring
  double *gcs;             // GLOBAL_SoundSpeed (ring means of cs)
  const double *p15;       // pow(Rmed, 1.5)
  const double *dxrad, *dxtheta, *invdxtheta, *mindx2;
  const double *dxtheta_cfl; // Rmed*(PMAX-PMIN)/ns as ConditionCFL forms it (SourceEuler.c:1344)
  const double *supp_torque;
  const double *sigmamed, *energymed, *vthetamed, *vradmed;
  const double *betatab;   // ComputeBetaCooling(Rmed)
  // TEMPPRESC: per ring the relaxation time (PrescTimeMed, or PRESCTIME0 /
  // Omega without VISCOSITY), SourceEuler.c:1162-1168
  int temppresc;
  const double *presc;
  const double *damp_lam;  // damping*damping per ring (0 outside the zones)
  const double *damp_tau;  // DAMPINGTODYNAMICALTIMERATIO*pow(Rmed,1.5)
  const int *damp_rings;   // list of rings inside the wave-killing zones
  int n_damp_rings;
  double vh_l1, vh_l2;     // log(r/rip), log(rip/ri2p) for ViscHeat at i=0
  // CFL / reductions
  double *ringmin, *vmoy;
  double *vt_part;  // beta cooling: per ring, SubStep2's partial sums of vtheta (one per CTA)
  double *partials;
  int n_partial_blocks;
  fb_ctl *ctl;
  // scalars
  double pmin, pmax, dphi, invdphi, omega_frame;
  // frame corotating with the first planet (FRAME C): OmegaFrame changes
  // every substep and lives in the control block; kernels read it via omf()
  int corot;
  double gamma, alpha, nu_const;
  int visc_mode;           // 0 inviscid, 1 alpha, 2 constant nu
  int energy, viscous_heating, beta_cooling, fast_transport;
  int wall, evanescent, add_floors, damp_axi, zero_vrad;
  // open and non-reflecting edges (SideEuler.c:300-410, 569-794) and the
  // constants they take from the 1-D tables (glibc pow on the host):
  // sqrt(Rmed2/Rmed1), sqrt(Rmed2/Rmed0), pow(Rmed[nr-1]/Rmed[nr-2], -0.5),
  // pow(Rinf[1], -1.5), pow(Rinf[nr-2], -1.5), the initial sound speeds of
  // rings 0 and 1 (adiabatic), SIGMASLOPE, Radii[0] and Radii[nr]
  int open_inner, kn_open, non_reflecting;
  double *edge_buf;  // 3 nsec: the non-reflecting edges' copies, read before written
  // thermal cooling (SourceEuler.c:1201-1290): the opacity field, set once
  // from the uploaded state as InitEuler sets it (SourceEuler.c:275), and
  // the Stefan-Boltzmann constant in code units (LowTasks.c:215)
  int thermal_cooling;
  double *opacity;
  double sigma_sb;
  // stellar irradiation: 0 none, 1 background temperature (irr_ring[i] =
  // its value at Rmed[i]), 2 imposed luminosity (irr_ring[i] =
  // Lstar/4/pi/Rmed[i]/Rmed[i])
  int irradiation;
  const double *irr_ring;
  double ob_vt1, ob_vt0, ob_vtout, nrb_om1, nrb_omn2, nrb_csinit0, nrb_csinit1, sigmaslope;
  double radii0, radiin;
  double floordens, wkzrmin, wkzrmax;
  int indirect_term, discard_gas_it, alt_gas_it, exclude_hill, roche, forced_circular;
  double indirect_smoothing, rochesmoothing, thicksmoothing, aspectratio, flaringindex;
  double masstaper;
  int self_gravity;
  int transport_only;      // stage test: Transport without floors/boundaries
  // Lagrangian particles: grids the gas substep leaves for the next particle
  // update (IndPotential, RadGradP, AziGradP, RadIndAcc, AziIndAcc,
  // RadSGAcc, AziSGAcc of src/SourceEuler.c:210-216); NULL without particles
  double *indpot, *rgp, *agp, *rind, *aind, *rsga, *asga;
  int particles, dust_feel_planets, dust_feel_disk;
  // DUSTFEEDBACK: the substep is also bounded by half the particles' minimum
  // stopping time (SourceEuler.c:1501-1507); NULL otherwise
  const double *dust_min_ts;
  // turbulent potential (MHD L): modes, their azimuthal factors
  // cos/sin(m Azimuth[j]) (2 x nm x ns, recomputed for redrawn modes) and
  // radial envelopes mygamma/r xi exp(-(r-rc)^2/sigma^2) (nm x nr)
  int lsa, lsa_nm, lsa_highm;
  double lsa_gamma, lsa_speedup, lsa_rmin, lsa_rmax, cav_rmin, cav_rmax, cav_ratio;
  fb_lsa *lsa_st;
  double *lsa_cs, *lsa_g;
  // thermal diffusion (energy equation): entropy diffusion (DIFFUSIVITY),
  // radiative diffusion 1 explicit / 2 implicit; per-cell scratch: the
  // entropy logarithm, the temperature (TempInt, updated in place by the
  // solver), the diffusion coefficient K or chi, the two explicit source
  // fields, the solver's coefficients a..f (6 fields), per-CTA residual
  // partial sums and the solver's grid barrier {count, generation}
  int ent_diff, rad_diff;
  double diffusivity;
  double *td_s, *td_t, *td_k, *td_ent, *td_rad, *sor_c[6], *sor_part;
  unsigned int *sor_bar;
  int sor_grid;
  // ComputeOpacities' constants (SourceEuler.c:1608-1701), for the opacity
  // of the current state at every substep when radiative diffusion is on
  int op_constant;
  double op_imposed, op_factor, op_utemp, op_umass, op_invl3, op_conv;
  // launch shapes (tuning): per-cell CTA width, cells per thread of the
  // azimuthal pass (0 = automatic), columns per CTA and rings per CTA of the
  // radial pass (0 = automatic), variant of the azimuthal pass (0 automatic,
  // 1 narrow, 2 wide, 3 packed, 4 register, 5 staged, 6 tile)
  int cell_bs, azi_E, rad_tx, rad_chunk, azi_variant;
};

// OmegaFrame as the current substep sees it: the control block's in a
// corotating frame (updated by the planets' step), else the constant
static __device__ __forceinline__ double omf(const KP &k) { return k.corot ? k.ctl->omega_frame : k.omega_frame; }

// Device state of the particles' random stream (src/DustUpdate.c:438-485).
// a / d rounded to nearest, given r = 1/d rounded to nearest (fb_rcp in the
// parity build): y = RN(a r) is
// within one ulp of a/d, its remainder a - d y is exact in one fma, and
// RN(y + r (a - d y)) = RN(a / d) (Markstein's theorem: P. Markstein, IBM J.
// Res. Dev. 34(1), 1990; J.-M. Muller et al., Handbook of Floating-Point
// Arithmetic, ch. 4).  Valid away from overflow and underflow.  Lets several
// quotients by one divisor share a single division.
static __device__ __forceinline__ double fb_quot(double a, double d, double r)
{
  const double y = a * r;
  const double e = fma(-d, y, a);
  return fma(e, r, y);
}

// Quotient of a van Leer slope, dq+ dq- / (dq+ + dq-), taken only where
// dq+ dq- > 0 (so the divisor is non-zero and of the numerator's sign).
// Parity build: the exact (IEEE, correctly rounded) division of the
// reference.  Fast build (FB_FAST): the hardware's approximate reciprocal
// (PTX rcp.approx.ftz.f64) refined by two Newton-Raphson steps,
// r <- r + r (1 - b r), each of which doubles the correct bits, then one
// product: a few ulp from the exact quotient, without the division's
// range-check branch.
static __device__ __forceinline__ double fb_vl_quot(double a, double b)
{
#if FB_FAST
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
  double e = fma(-b, r, 1.0);
  r = fma(r, e, r);
  e = fma(-b, r, 1.0);
  r = fma(r, e, r);
  return a * r;
#else
  return a / b;
#endif
}

// 1/d for the shared-divisor quotients fb_quot.  Parity build: correctly
// rounded (IEEE division), which makes fb_quot exact.  Fast build: the
// approximate reciprocal refined by two Newton-Raphson steps (a few ulp), so
// that fb_quot is within a few ulp of the quotient.
static __device__ __forceinline__ double fb_rcp(double d)
{
#if FB_FAST
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
#else
  return 1.0 / d;
#endif
}

// The van Leer slope of the azimuthal pass from the differences dq- and dq+
// of a quantity across a cell, times invdx: dq+ dq- / (dq+ + dq-) invdx where
// dq+ dq- > 0, else 0 (TransportEuler.c:392-433).  The fast build evaluates
// the quotient in every lane and selects afterwards, so that the slopes of a
// thread's cells run side by side instead of behind a branch each.
static __device__ __forceinline__ double fb_vl_slope(double dqm, double dqp, double invdx)
{
#if FB_FAST
  const double num = dqp * dqm;
  const double v = fb_vl_quot(num, dqp + dqm) * invdx;
  return (num > 0.0) ? v : 0.0;
#else
  return (dqp * dqm > 0.0) ? fb_vl_quot(dqp * dqm, dqp + dqm) * invdx : 0.0;
#endif
}

// Kernel launches of the step.  With programmatic dependent launch a
// kernel may be scheduled while the one before it in the stream drains;
// every kernel of the step starts with fb_grid_dependency(), which waits
// until the previous grid has completed and its writes are visible, then
// lets the next grid be scheduled (it only starts once every CTA of this
// grid has started, so it never takes resources this grid still needs).
extern int fb_pdl;  // 1: launches carry the programmatic-serialization attribute
template <typename... KArgs, typename... Args>
static inline void fb_launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             Args... args)
{
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = fb_pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}
static __device__ __forceinline__ void fb_grid_dependency()
{
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

struct fb_dust_ctl {
  unsigned long long x;        // drand48 state after the last draw
  long long kicks;             // calls made so far by each Gaussian generator
  double carry_rad, carry_phi; // their cached second deviates (kicks odd)
  long long t_start, c_last;   // first pair event of this substep, last candidate used
  int K, npairs, err, pad;     // kicked particles, accepted pairs needed, shortfall flag
  double min_ts;               // Minimum_Stopping_Time of the last interpolation (Dsys.c:336,758)
  // per planet, for the substep's velocity update (DustUpdate.c:342-352):
  // radius, azimuth and smoothing length, the same for every particle
  double pl_r[FB_MAX_PLANETS], pl_t[FB_MAX_PLANETS], pl_eps[FB_MAX_PLANETS];
};

// Particle arrays (structure of arrays in the reference's index order) and
// the constants of the particle update, passed by value.
struct PP {
  int n, ncand;
  double *r, *th, *vr, *vth, *l, *size, *st;
  int *flag, *kidx, *kick_bsum, *cand_flag, *cand_bsum;
  double2 *pairs;
  fb_dust_ctl *dc;
  const double *azimuth, *aziinf;  // ns
  double aziinf0, azisupl, delta_r, delta_phi;
  double rmin, rmax, unit_mass, inv_unit_length2, dust_density_cu;
  double aspectratio, thicksmoothing, flaringindex;
  int log_grid, feel_disk, feel_planets, feel_sg, feel_turb, sfta;
  int restokes;  // WRITEDUSTDENSITY: interpolation again after the update (SourceEuler.c:526-531)
  // Storage order: once per DT the particles are moved into cell order (a
  // counting sort), so that a warp's grid gathers hit neighbouring cells and
  // its particle loads and stores stay coalesced.  orig[slot] is the
  // reference's index of the particle in a slot: the random stream and the
  // downloads follow it; no result depends on the storage order.
  int *orig, *perm, *key, *cell_count, *cell_bsum;
  double *pscratch;  // 7 n doubles: the moved arrays
  int *oscratch;     // n: the moved orig
  int ncells;        // nr*ns + 1 (the last bucket holds particles off the grid)
  // first guess of a particle's ring from the grid law (log or arithmetic),
  // corrected exactly against the radii
  double ring_r0, ring_inv_r0, ring_inv_step;
  // log of the interface and centre radii (glibc log on the host): the fast
  // build takes a TSC weight's |log(rp / R)| as |log rp - log R|
  const double *log_rinf, *log_rmed;
};

// launchers (fb_gas.cu)
void fb_launch_cfl(const KP &k, cudaStream_t s);
void fb_launch_planets(const KP &k, const PP *pp, cudaStream_t s);
void fb_launch_correct_vtheta(const KP &k, cudaStream_t s);  // corotating frame: CorrectVtheta
void fb_launch_soundspeed(const KP &k, int update_gcs, cudaStream_t s);
void fb_launch_potential(const KP &k, cudaStream_t s);
// turbulent potential: mode draws and tables after the controller, the
// modes' sum added to the potential after k_potential (two and one launches)
void fb_launch_lsa_modes(const KP &k, cudaStream_t s);
void fb_launch_lsa_add(const KP &k, cudaStream_t s);
// thermal diffusion: the opacity of the current state (before the CFL
// kernel with explicit radiative diffusion) and SubStep0 after the
// controller; each returns its kernel launches
int fb_launch_opacity_now(const KP &k, cudaStream_t s);
int fb_launch_substep0(const KP &k, cudaStream_t s);
int fb_launch_td_cfl(const KP &k, cudaStream_t s);  // explicit radiative diffusion's CFL limits
int fb_sor_grid(void);  // CTAs of the solver kernel the GPU holds at once
void fb_launch_substep1(const KP &k, cudaStream_t s);
void fb_launch_viscous_terms(const KP &k, const double *vr, const double *vt, cudaStream_t s);
void fb_launch_viscous_update(const KP &k, double *vr, double *vt, double dt_override, cudaStream_t s);
void fb_launch_substep2(const KP &k, cudaStream_t s);
void fb_launch_substep3(const KP &k, cudaStream_t s);
void fb_launch_transport(const KP &k, double dt_override, cudaStream_t s);
void fb_launch_transport_radial(const KP &k, double dt_override, cudaStream_t s);
// vmed_done: the tile variant's ring means are already taken (fb_launch_azi_vmed)
void fb_launch_transport_azimuthal(const KP &k, double dt_override, cudaStream_t s, bool vmed_done = false);
int  fb_launch_azi_vmed(const KP &k, double dt_override, cudaStream_t s);
void fb_launch_transport_vr(const KP &k, cudaStream_t s);
void fb_launch_edges(const KP &k, cudaStream_t s);  // open / non-reflecting edges
// ComputeOpacities (SourceEuler.c:1608-1701) of the current state:
// constant = SETCONSTANTOPACITY; conv = 0.1 unit_length^-2 unit_mass
void fb_launch_opacity(const KP &k, int constant, double imposed, double factor, double unit_temperature,
                       double unit_mass, double inv_l3, double conv, cudaStream_t s);
void fb_launch_floors_boundary(const KP &k, cudaStream_t s);
void fb_launch_damping(const KP &k, double dt_override, cudaStream_t s);
void fb_launch_diag(const KP &k, double *out2, cudaStream_t s);
void fb_launch_derived(const KP &k, int which, double *out, cudaStream_t s);
void fb_launch_boundary_only(const KP &k, cudaStream_t s);
int  fb_gas_prepare(int ns, int energy);  // kernel attributes (shared memory); loads the azimuthal kernels
int  fb_transport_preload(void);          // loads the radial and vr transport kernels
// launch-shape candidates the tuner may try (fb_gas.cu)
int  fb_azi_E_valid(int ns, int energy, int E);   // 1 if E cells/thread fit this ring
int  fb_azi_E_auto(int ns);
int  fb_azi_launches(const KP &k);  // kernel launches of one azimuthal pass
int  fb_azi_variant(int ns, int energy, int E, int variant);  // variant a launch takes (0: cannot run)
int  fb_rad_chunk_auto(const KP &k);
int  fb_rad_chunks_balanced(const KP &k, int tx, int *out, int max);
int  fb_allow_max_dynamic_smem(const void *func);
void fb_launch_begin_dt(const KP &k, double DT, cudaStream_t s);
void fb_launch_loop_cond(const KP &k, cudaGraphConditionalHandle h, int cap, cudaStream_t s);
// self-gravity (fb_sg.cu)
struct fb_sg;
int  fb_sg_create(fb_sg **out, const fb_params *p, const fb_geom *g, cudaStream_t s);
void fb_sg_destroy(fb_sg *sg);
void fb_sg_accel(fb_sg *sg, const KP &k, const double *dens, cudaStream_t s);
// refresh = 1: the Dt = 0 call of main.c:316 on Vrad/Vtheta (fields only)
void fb_sg_update_velocities(const KP &k, cudaStream_t s, int refresh = 0);
// context accessors for the other modules (fb_api.cu)
const KP *fb_ctx_kp(const fb_ctx *ctx);
KP *fb_ctx_kp_mut(fb_ctx *ctx);
cudaStream_t fb_ctx_stream(const fb_ctx *ctx);
void fb_ctx_count_launches(fb_ctx *ctx, int n);
// diagnostics (fb_diag.cu)
void fb_launch_vortensity(const KP &k, double *xi, cudaStream_t s);
void fb_launch_body_force(const KP &k, double x, double y, double rsmoothing, double cutoff, double *part,
                          cudaStream_t s);
void fb_launch_ring_mean(const double *f, int nr, int ns, double *out, cudaStream_t s);
// Lagrangian particles (fb_dust.cu)
void fb_launch_dust_substep(const KP &k, const PP &pp, cudaStream_t s, cudaEvent_t planets_done);
void fb_launch_dust_interpolation_only(const KP &k, const PP &pp, cudaStream_t s);
int  fb_dust_launches(const PP &pp);
int fb_launch_dust_sort(const KP &k, const PP &pp, cudaStream_t s);  // returns launches
void fb_launch_dust_iota(const PP &pp, cudaStream_t s);
void fb_launch_dust_to_reference_order(const PP &pp, const double *src, double *dst, cudaStream_t s);
int  fb_sg_launches(const fb_sg *sg);  // kernels per fb_sg_accel + update
void fb_sg_rows_fwd(fb_sg *sg, const KP &k, const double *dens, cudaStream_t s);
void fb_sg_cols(fb_sg *sg, cudaStream_t s);
void fb_sg_rows_inv(fb_sg *sg, const KP &k, const double *dens, cudaStream_t s);
