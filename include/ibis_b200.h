/* C ABI of the B200-native IBIS 3.0 hourly land-surface step.
 *
 * The reference exposes this path as one pure function over Equinox pytrees,
 *     timestep_body(state, consts, params, dtime) -> state
 * (python-port/ibis/timestepping/loops.py:234-284), scanned by the day loop
 * _run_day_inner._step_body (python-port/ibis/timestepping/loops_gswp3.py:115-320).
 * It has no operator, plugin or FFI layer of its own; these entry points are
 * what an XLA FFI handler or a ctypes/cgo binding of that function calls.
 *
 * Conventions
 *   - All buffer pointers are DEVICE pointers owned by the caller.
 *   - Buffers are structure-of-arrays "planes" (include/ibis_layout.h):
 *     element (plane p, cell i) is buf[p * ld + i]; ld >= ncell, ld % 32 == 0.
 *   - Calls are asynchronous on `stream` (a cudaStream_t; NULL = legacy default).
 *   - Return 0 on success, -EINVAL for bad arguments, or a value <= -1000
 *     (-(cudaError_t) - 1000) when the launch itself failed.
 *   - A column whose state becomes non-finite is data, not an error: the kernel
 *     sets status[0] |= 1 and status[1] = min(status[1], cell).  `status` may be
 *     NULL; otherwise it is a device int[2] the caller initialises to {0, INT_MAX}.
 */
#ifndef IBIS_B200_H
#define IBIS_B200_H

#include "ibis_layout.h"

#ifdef __cplusplus
extern "C" {
#endif

/* nstep hourly steps of timestep_body (+ the day-loop accumulators when the
 * IBIS_FLAG_ACC / _CH4 / _SOIL_MEANS bits of params->flags are set) on ncell
 * columns, in FP32 with FP64 canopy and soil-water solves.
 *   prog   [IBIS_PROG_COUNT][ld]              in/out: prognostic state
 *   stat   [IBIS_STAT_COUNT][ld]              in: per-cell static inputs
 *   forc   [nstep][IBIS_FORC_COUNT][ld]       in: hourly forcing (the atm leaves)
 *   diag   [IBIS_DIAG_COUNT][ld] or NULL      out: last step's diagnostics (IBIS_FLAG_DIAG)
 *   acc    [2*IBIS_ACC_COUNT][ld] or NULL     in/out: accumulators then Kahan terms
 * Replaces: timestep_body (loops.py:234) iterated by _step_body (loops_gswp3.py:115). */
int ibis_step_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc, int ncell, int ld,
                  int nstep, const IbisParams* params, int* status, void* stream);

/* Same contract as ibis_step_f32, run as two kernels per hour: a surface
 * phase (radiation, interception, canopy solve) and a ground phase (snow,
 * soil, accumulators) that hand ibis_mid_planes() values per cell to each
 * other through `scratch` [ibis_mid_planes()][ld] (device, caller-owned).
 * Each kernel needs fewer registers than the fused one; which form is faster
 * depends on the batch (see ibis_b200/tune.py).
 * Replaces: timestep_body (loops.py:234) iterated by _step_body (loops_gswp3.py:115). */
int ibis_step_split_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc, float* scratch,
                        int ncell, int ld, int nstep, const IbisParams* params, int* status, void* stream);

/* Number of scratch planes ibis_step_split_f32 needs. */
int ibis_mid_planes(void);

/* ibis_step_f32 / ibis_step_split_f32 with an explicit launch configuration
 * (0 <= config < ibis_num_configs()): the form (fused or two-kernel), block
 * size and register budget.  `scratch` is required by two-kernel configs and
 * ignored by fused ones.  ibis_b200/tune.py times them and picks one per batch.
 * Every configuration exists for the F77 canopy without the sunlit/shaded
 * split; other flag sets have configurations 0 and 8 (and 6 for the IBIS 3.0
 * kernels with both canopies of one kind), and any other fused (two-kernel)
 * configuration runs as 0 (8) for them.
 * Replaces: timestep_body (loops.py:234) iterated by _step_body (loops_gswp3.py:115). */
int ibis_step_config_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc, float* scratch,
                         int ncell, int ld, int nstep, const IbisParams* params, int* status, void* stream,
                         int config);

/* Launch configurations: count, and the description of one
 * (form 0 = fused, 1 = two-kernel, 2 = fused with each hour's forcing tile
 * brought into shared memory by bulk copies while the hour before it runs;
 * block sizes and min resident blocks/SM).  A form-2 launch whose forcing
 * pointer is not 16-byte aligned runs the form-0 kernel of the same block
 * size; one whose bounded wait for a copy gave up sets status[0] bit 2
 * (value 4), and its results are not to be used. */
int ibis_num_configs(void);
int ibis_config_info(int config, int* form, int* block, int* min_blocks, int* block2, int* min_blocks2);

/* ibis_step_split_f32 for callers that cannot allocate device memory (an XLA
 * custom-call handler, which must not allocate behind XLA's own allocator; a
 * serving loop that reserved all device memory up front and has none left to
 * hand out).  No counterpart in the reference: the
 * hand-off planes live in a fixed array inside this library, sized for at most
 * 32768 cells (ld <= 32768, 3.5 MiB held on every GPU that loads the library
 * until the process exits); larger ld returns -EINVAL with a message on stderr.
 * No cudaMalloc, cudaFree or other allocating call is made.  The first call on
 * each device looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture; the cached address is not
 * refreshed after cudaDeviceReset.  Every call on a device
 * shares the one array and it keeps the last call's contents; the surface
 * kernel writes every value the ground kernel reads, so nothing needs
 * clearing, but calls that overlap on the GPU (different streams, or
 * different host threads) race on it and must be serialised by the caller. */
int ibis_step_split_noalloc_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc,
                                int ncell, int ld, int nstep, const IbisParams* params, int* status, void* stream);

/* ibis_step_f32 with the forcing in HOST memory and the prognostic state read
 * back to HOST memory, for callers whose inputs start and end on the host (the
 * reference's timestep_body called on NumPy state, a day loop fed from files).
 * The copies overlap the steps on streams of the library's own:
 *   - a batch of more than 1.15 waves of the launch configuration is cut into
 *     groups of columns (`group` cells, a multiple of 32; 0 = a sixteenth of
 *     ncell, rounded up to whole blocks of the launch configuration; raised
 *     so there are at most 64 groups), each
 *     group's forcing copied in, stepped and its state copied out while other
 *     groups step;
 *   - a smaller batch (group 0) is one group whose hours are cut into chunks,
 *     each chunk's copy overlapping the steps of the chunk before.
 *   `chunk` sets the hours per chunk: c > 0 equal chunks of c hours; -c, c
 *   hours then the rest; 0, for several groups a third of the hours then the
 *   rest (all groups' first chunks are copied before any group's second), for
 *   one group 4 hours growing by 1.75 per chunk; groups x chunks <= 256.
 *   host_forc  [nstep][IBIS_FORC_COUNT][ld]  pinned HOST: hourly forcing
 *   forc       [nstep][IBIS_FORC_COUNT][ld]  DEVICE: where the forcing lands
 *   host_prog  [IBIS_PROG_COUNT][ld] pinned HOST, or NULL: the state after the
 *              last hour (device prog is updated either way)
 *   config     -1 (ibis_step_f32's choice) or a fused launch configuration
 *   other arguments as for ibis_step_f32; status[1] counts cells from 0 over
 *   all groups.
 * Everything queued on `stream` before the call runs first, and work queued on
 * it afterwards (a read of host_prog after a stream synchronise) runs after
 * every group's hours and copies.  Calls from several host threads are
 * serialised by the library (they share its streams).
 * Replaces: timestep_body (loops.py:234) iterated by _step_body (loops_gswp3.py:115)
 * on host arrays. */
int ibis_step_host_f32(float* prog, const float* stat, const float* host_forc, float* forc, float* diag, float* acc,
                       float* host_prog, int ncell, int ld, int nstep, const IbisParams* params, int* status,
                       int group, int chunk, int config, void* stream);

/* Days of the step from daily weather in HOST memory, the state read back to
 * HOST memory: per group of columns (`group` as for ibis_step_host_f32, but
 * 0 = a twentieth of ncell in whole blocks), the
 * group's daily weather copied in, its hourly forcing generated on the device
 * (as ibis_diurnal_f32 generates it, the variates keyed by each cell's index
 * in the caller's numbering, so the forcing equals one call over all cells),
 * its nday * 86400/dtime hours stepped and its state copied out, on streams of
 * the library's own so one group's work overlaps the others'.
 *   host_daily [nday][IBIS_DAILY_COUNT][ld]  pinned HOST: daily weather
 *   daily      [nday][IBIS_DAILY_COUNT][ld]  DEVICE: where it lands
 *   lat        [ld] DEVICE: latitude (degrees)
 *   forc       [nday * 86400/dtime][IBIS_FORC_COUNT][ld] DEVICE: the generated forcing
 *   jday0, day0, seed, dflags as for ibis_diurnal_f32 (dtime from params);
 *   other arguments as for ibis_step_host_f32.
 * Replaces: _run_day_inner's days -- compute_precip_timing + diurnal
 * (python-port/ibis/physics/weather.py:395-601) and timestep_body / _step_body
 * (loops_gswp3.py:115-320) -- on host arrays. */
int ibis_day_host_f32(float* prog, const float* stat, const float* host_daily, float* daily, const float* lat,
                      float* forc, float* diag, float* acc, float* host_prog, int ncell, int ld, int nday, int jday0,
                      int day0, unsigned int seed, unsigned int dflags, const IbisParams* params, int* status,
                      int group, int config, void* stream);

/* A calibration ensemble: nrun runs, each one parameter vector at one site
 * over its own record of hourly forcing.  Per-run buffers use ld_run, per-site
 * buffers ld_site (both multiples of 32, >= the count).
 *   prog        [IBIS_PROG_COUNT][ld_run]       in/out: state of every run
 *   acc         [2*IBIS_ACC_COUNT][ld_run]/NULL in/out: accumulators + Kahan terms
 *   stat        [IBIS_STAT_COUNT][ld_site]      in: static inputs of every site
 *   forc        [forc_len][IBIS_FORC_COUNT]     in: hourly forcing records (16-byte aligned)
 *   run_params  [IBIS_RUN_COUNT][ld_run]        in: calibration vector of every run
 *   run_site    [nrun]  site of the run; run_forc [nrun] index of its first record
 *   run_nstep   [nrun]  hours in its record (records run_forc .. run_forc+nstep-1)
 *   run_pos     [nrun] or NULL: hours each run completed before this call (its
 *               records start at run_forc regardless; run_pos only places the
 *               year ends of the yearly totals), NULL = 0
 *   order       [norder] or NULL: the runs to advance, in the order they are
 *               taken (longest first is best); NULL = all nrun runs in index order
 *   norder      entries of order (ignored when order is NULL)
 *   yearly      [nyear][IBIS_YEARLY_COUNT][ld_run] or NULL: running totals of the
 *               IBIS_YEARLY accumulators at the end of each year_steps hours
 *   queue       device int used as the work counter (reset by the call)
 *   status      device int[2] as for ibis_step_f32; bit 1 (value 2) flags a run
 *               whose descriptor is out of range, which is then skipped.
 * No counterpart in the reference's step API: its calibration harness runs
 * one site at a time in host worker processes (verify/calibration/site_fit.py:375-436). */
typedef struct IbisEnsemble {
    float* prog;
    float* acc;
    const float* stat;
    const float* forc;
    const float* run_params;
    const int* run_site;
    const long long* run_forc;
    const int* run_nstep;
    const int* run_pos;
    const int* order;
    float* yearly;
    long long forc_len;
    int nrun, ld_run, nsite, ld_site, nyear, year_steps, norder;
    int* queue;
    int* status;
} IbisEnsemble;

/* Every run of the ensemble from its first hour to its last in ONE persistent
 * launch: grid = SMs x resident blocks of `block` threads (a multiple of 32,
 * <= 256; 0 picks one from the run count), each warp drawing 32 runs at a time
 * from the work counter.  params->flags selects the model variants and the
 * accumulators as for ibis_step_f32 (no diagnostics), the IBIS_FLAGS_X3
 * switches included: a run's vector replaces the parameters it carries, and
 * the switches' own tables (coefm_pft, the acclimation tables, crop scales)
 * come from params. */
int ibis_ensemble_f32(const IbisEnsemble* ens, const IbisParams* params, int block, void* stream);

/* The same runs advanced `nhour` hours in nhour launches (one per hour), from
 * the hour held in the device int *hour, which the last launch advances by
 * nhour: a fixed sequence that can be captured once in a CUDA graph and
 * replayed until every record has ended.  Every run r < nrun whose record
 * covers the hour takes its step (order is not used). */
int ibis_ensemble_hours_f32(const IbisEnsemble* ens, const IbisParams* params, int* hour, int nhour,
                            void* stream);

/* The daily-weather form of an ensemble: instead of hourly records, every
 * site has day records and each run generates its hours as it steps, from the
 * reference's diurnal algorithm (as ibis_diurnal_f32 does for columns), so a
 * site-day costs 48 bytes of forcing instead of 24 x 48.
 *   records   [len][12]: the IBIS_DAILY_* words of the day, its day of year
 *             (1..366, as a float) at word IBIS_DAILY_COUNT, two padding words;
 *             16-byte aligned
 *   site_lat  [nsite] latitude (degrees)
 *   seed      key of the counter-based variates, drawn per (seed, record, site)
 *   flags     IBIS_DIURNAL_OBSERVED_FIRA: longwave from the fira word
 * With this form ens->run_forc[r] is the run's first day record, ens->forc and
 * ens->forc_len are not used, and a run's hours start at midnight of that day. */
typedef struct IbisEnsembleDaily {
    const float* records;
    const float* site_lat;
    long long len;
    unsigned int seed;
    unsigned int flags;
} IbisEnsembleDaily;

/* ibis_ensemble_f32 over day records (IbisEnsembleDaily) instead of hourly ones.
 * Replaces: the calibration harness's per-site runs of the day loop, which
 * disaggregate each day with compute_precip_timing + diurnal
 * (python-port/ibis/physics/weather.py:395-601; loops_gswp3.py:115-124). */
int ibis_ensemble_daily_f32(const IbisEnsemble* ens, const IbisEnsembleDaily* daily, const IbisParams* params,
                            int block, void* stream);

/* Resident blocks per SM of the persistent ensemble kernel at `block` threads,
 * for the variant params->flags selects (0 when it cannot run). */
int ibis_ensemble_occupancy(const IbisParams* params, int block);

/* Hourly forcing from daily weather on the device: for each of nday days and
 * each hour of the day (86400 / dtime hours), the FORC planes of that hour.
 *   daily  [nday][IBIS_DAILY_COUNT][ld]   in: daily weather (IBIS_DAILY_* planes)
 *   lat    [ld]                           in: latitude (degrees)
 *   forc   [nday * 86400/dtime][IBIS_FORC_COUNT][ld]  out: hourly forcing, the
 *          layout ibis_step_f32 reads
 * Day d is day of year ((jday0 - 1 + d) mod 365) + 1 and draws its variates
 * (event length and start, hourly wind) from a counter-based generator keyed by
 * (seed, day0 + d, cell), so any day of any cell regenerates independently.
 * flags: IBIS_DIURNAL_OBSERVED_FIRA takes the longwave from the fira plane.
 * Replaces: compute_precip_timing + diurnal (python-port/ibis/physics/weather.py:395-601),
 * called once per day and hour by _run_day_inner (loops_gswp3.py:115-124). */
#define IBIS_DIURNAL_OBSERVED_FIRA 1u
int ibis_diurnal_f32(const float* daily, const float* lat, float* forc, int ncell, int ld, int nday, int jday0,
                     int day0, float dtime, unsigned int seed, unsigned int flags, void* stream);

/* ibis_diurnal_f32 with an observed hourly shortwave total where a cell-day
 * has one: sw_obs [nday][86400/dtime][ld] (W m-2 at each hour), use [nday][ld]
 * (nonzero: that cell-day uses it).  Where used, the total is split into direct
 * and diffuse by the hourly clearness-index relation of Spitters et al. (1986)
 * and into the two bands; elsewhere the generator's shortwave stands.
 * Replaces: observed_shortwave (python-port/ibis/physics/weather.py:458-481), applied
 * per hour by _run_day_inner (loops_gswp3.py:126-129). */
int ibis_diurnal_sw_f32(const float* daily, const float* lat, const float* sw_obs, const unsigned char* use,
                        float* forc, int ncell, int ld, int nday, int jday0, int day0, float dtime, unsigned int seed,
                        unsigned int flags, void* stream);

/* Daily cadence of the day loop, one thread per cell, around a day's hourly
 * steps (ibis_step_* with accumulators, fed by ibis_diurnal_f32 or by the
 * caller's forcing):
 *   stat   [IBIS_STAT_COUNT][ld]      frac, lai, ztop, zbot (begin), tco2mic (end)
 *   dayst  [IBIS_DAYST_COUNT][ld]     phenology, 10-day means, annual sums,
 *                                     litter and soil carbon pools (IBIS_DAYST_*)
 *   acc    [2 * IBIS_ACC_COUNT][ld]   the step's accumulators with their
 *                                     compensation planes
 *   td     [ld]                       the day's mean air temperature (K)
 *   prog   [IBIS_PROG_COUNT][ld]      soil temperature, water and ice (end)
 * ibis_day_begin: phenology from the standing 10-day means and the last hour's
 * soil-water stress (IBIS_ACC_STRESSTU_LAST / _STRESSTL_LAST), then the daily
 * sums (adrain, adsnow, adaet, a10anc*) zeroed.
 * ibis_day_end: 10-day means and annual sums from the daily sums, the
 * decomposition factors, one day of soil C/N and the respiration sums.
 * params supplies hsoi, ndaypy and epsilon; dayparams the phenology and
 * soil-biogeochemistry constants.  Arithmetic is double for both buffer types.
 * With dayparams->seasonal_on = 1, ibis_day_begin first advances the seasonal
 * states (acclim_x, ssen_u, ssen_l; day length from the latitude plane and
 * dayparams->jday) and gates phenology by photoperiod where sen_photoperiod_*
 * is 1; with stress_on = 1, ibis_day_end adds the last hour's stress to the
 * growing-season sums (aystressu, aystressl, stress_nday).  Switches other
 * than 0 or 1 return -EINVAL.
 * Replaces: the per-day body of _run_month_scan._day_body
 * (python-port/ibis/timestepping/loops_gswp3.py:382-437, 466-596), with
 * pheno (physics/phenology.py:89-287) and soilbgc (physics/biogeochem.py:23-243). */
int ibis_day_begin_f32(float* stat, float* dayst, float* acc, const float* td, int ncell, int ld,
                       const IbisParams* params, const IbisDayParams* dayparams, void* stream);
int ibis_day_begin_f64(double* stat, double* dayst, double* acc, const double* td, int ncell, int ld,
                       const IbisParams* params, const IbisDayParams* dayparams, void* stream);
int ibis_day_end_f32(const float* prog, float* stat, float* dayst, const float* acc, const float* td, int ncell,
                     int ld, const IbisParams* params, const IbisDayParams* dayparams, void* stream);
int ibis_day_end_f64(const double* prog, double* stat, double* dayst, const double* acc, const double* td,
                     int ncell, int ld, const IbisParams* params, const IbisDayParams* dayparams, void* stream);

/* Monthly wetland methane around a month of days (one thread per cell):
 *   wet    [IBIS_WET_COUNT][ld]     flux, annual, zwt (the MethaneState leaves),
 *                                   rh0 (ayco2mic at the month's start), ch4c
 *                                   (the year's CH4 carbon taken out of Rh)
 *   acc    [2 * IBIS_ACC_COUNT][ld] the step's accumulators (IBIS_ACC_CH4: the
 *                                   sum of the day means of the hourly flux)
 *   dayst  [IBIS_DAYST_COUNT][ld]   ayco2mic (may be NULL unless partitioning)
 * ibis_month_begin: zero the CH4 accumulator, keep ayco2mic in rh0; with
 * IBIS_MONTH_NEW_YEAR clear annual and ch4c first (reset_annual).
 * ibis_month_end: the month's flux -- with IBIS_MONTH_FROM_MEAN the mean of
 * the hourly fluxes (methane_step_from_mean), else methane_flux of the
 * end-of-month state with Rh = tco2mic * 12e-3 * 86400 (methane_step) --, the
 * water table (observed where params->flags has IBIS_FLAG_ZWT_OBS and the
 * STAT zwt_obs plane is finite), annual += flux * ndays; then, if `scale`
 * (per-cell inundated fraction, [ld]) is not NULL, scale_month; then with
 * IBIS_MONTH_PARTITION the month's CH4 carbon (ch4_carbon_from_rh) is taken
 * out of ayco2mic and added to ch4c.
 * Replaces: methane_step / methane_step_from_mean / reset_annual / scale_month /
 * ch4_carbon_from_rh (python-port/ibis/bgc/methane.py:431-496) as the GSWP3
 * month driver calls them (timestepping/loops_gswp3.py:740-760). */
#define IBIS_MONTH_NEW_YEAR 1u
#define IBIS_MONTH_FROM_MEAN 2u
#define IBIS_MONTH_PARTITION 4u
int ibis_month_begin_f32(float* acc, float* wet, const float* dayst, int ncell, int ld, unsigned int flags,
                         void* stream);
int ibis_month_begin_f64(double* acc, double* wet, const double* dayst, int ncell, int ld, unsigned int flags,
                         void* stream);
int ibis_month_end_f32(const float* prog, const float* stat, const float* acc, float* wet, float* dayst,
                       const float* scale, int ncell, int ld, int ndays, const IbisParams* params,
                       unsigned int flags, void* stream);
int ibis_month_end_f64(const double* prog, const double* stat, const double* acc, double* wet, double* dayst,
                       const double* scale, int ncell, int ld, int ndays, const IbisParams* params,
                       unsigned int flags, void* stream);

/* ---------------------------------------------------------------------------
 * Wetland (inundated) area of the monthly methane: the two optional sources of
 * the month's fraction besides the WAD2M climatology.  Arithmetic in float64,
 * as the reference's host-side numpy.
 * ------------------------------------------------------------------------- */

/* Dynamic wetland area: f = clip(clip(fclim (1 + beta A), fmin, fmax), 0, 1),
 * A = (W - mu) / sd (0 where sd <= 1e-9 or the top layer is frozen), W the
 * liquid water of the top four layers (wsoi * poros * hsoi, a layer at or
 * below 273.16 K counting 0) of the state in `prog` / `stat`.
 *   area   [6][ld] double: fclim, mu, sd, beta, fmin, fmax of the month
 *   f_out  [ld] float: the month's fraction (e.g. the STAT f_inund plane)
 * Replaces: root_zone_water / dynamic_fraction (python-port/ibis/bgc/wetland_area.py:22-39)
 * as the global driver calls them (scripts/run_global.py:806-810). */
int ibis_wetland_dynamic_f32(const float* prog, const float* stat, const double* area, float* f_out, int ncell,
                             int ld, const IbisParams* params, void* stream);

/* The learned wetland's feature builder, one month per call: the 33 monthly
 * predictors in the model's order (DYN_FEATS) from the month's MEAN soil state
 * and its water totals, with the months it keeps for lags, 3-month means and
 * the 5 x 5 neighbourhood means (a box filter that wraps at every edge of the
 * nlat x nlon grid, as scipy's uniform_filter(mode='wrap')). */
#define IBIS_WETLAND_NFEAT 33
enum {
    IBIS_WFB_W = 0,        /* W of the last 4 months, oldest first */
    IBIS_WFB_PRCP = 4,     /* precipitation, 3 months */
    IBIS_WFB_RUNOFF = 7,   /* runoff + drainage, 3 months */
    IBIS_WFB_W3 = 10,      /* 3-month means of W, 4 months */
    IBIS_WFB_P3 = 14,      /* of precipitation, 4 months */
    IBIS_WFB_R3 = 18,      /* of runoff, 4 months */
    IBIS_WFB_NP3 = 22,     /* neighbourhood means of P3, 3 months */
    IBIS_WFB_NR3 = 25,     /* of R3, 3 months */
    IBIS_WFB_COUNT = 28
};
typedef struct IbisWetlandBuilder {
    int npoi, ld, nlat, nlon;
    const int* cell_i;     /* [npoi] device: grid row of each land point */
    const int* cell_j;     /* [npoi] device: grid column */
    const double* poros;   /* [4][ld] device: porosity of the top four layers */
    double hsoi[4];        /* thickness of the top four layers, m */
    double* lf;            /* [nlat*nlon] device: box filter of the land mask (ibis_wetland_grid) */
    double* buf;           /* [IBIS_WFB_COUNT][ld] device: months kept (in/out) */
    double* work;          /* [4][nlat*nlon] device: scratch */
    int nmonth;            /* months stepped before this call */
} IbisWetlandBuilder;

/* Fill b->lf: the box filter of the land mask (1 at the land points). */
int ibis_wetland_grid(const IbisWetlandBuilder* b, void* stream);

/* One month: means [19][ld] float (tsoi 6, wsoi 6, wisoi 6, tg), totals [3][ld]
 * float (precipitation, AET, runoff + drainage of the month); feats
 * [IBIS_WETLAND_NFEAT][ld] double out.  The caller increments b->nmonth after.
 * Replaces: FeatureBuilder.step (python-port/ibis/bgc/wetland_learned.py:75-104). */
int ibis_wetland_features(const IbisWetlandBuilder* b, const float* means, const float* totals, double* feats,
                          void* stream);

/* The trained models, one gradient-boosted tree ensemble per wetland band, in
 * flat node arrays (from XGBoost JSON boosters by ibis_b200/wetland.py): a
 * row goes left where its predictor is below `value` (float32), or, where it
 * is NaN, the way default_left says; a leaf's `value` is its output; a model's
 * prediction is base_margin plus its trees' leaves summed in float32, tree
 * after tree, then transform (0 identity, 1 logistic). */
typedef struct IbisForest {
    int nband, nfeat;
    const int* tree_first;            /* [nband + 1] device */
    const int* node_first;            /* [ntree + 1] device */
    const int* left;                  /* [nnode] device, -1 at a leaf */
    const int* right;                 /* [nnode] device */
    const int* feature;               /* [nnode] device */
    const float* value;               /* [nnode] device */
    const unsigned char* default_left;/* [nnode] device */
    const float* base_margin;         /* [nband] device */
    const int* transform;             /* [nband] device */
} IbisForest;

/* The learned fraction of one month: every land point gets clip(f_base, 0, 1),
 * then each cell p of the trained file (land point pts[p], band[p]) gets
 * clip(clip(fclim[p] + lam[band] (P - pbar[p]), 0, fmax[p]), 0, 1), P its
 * model's prediction (clipped to [0, 1]) on the 33 predictors of `feats` at
 * the point and the file's 12 static predictors.  Device arrays:
 *   pts, band [ncells] int;  fclim, pbar (the month's), fmax [ncells] double;
 *   stat [ncells][12] double;  lam [nband] double;  f_base, f_out [ld] float
 * Replaces: LearnedWetland.predict / fraction and hybrid_fraction
 * (python-port/ibis/bgc/wetland_learned.py:107-160). */
int ibis_wetland_learned(const IbisForest* forest, const double* feats, int npoi, int ld, const int* pts,
                         const int* band, const double* fclim, const double* pbar, const double* fmax,
                         const double* stat, const double* lam, int ncells, const float* f_base, float* f_out,
                         void* stream);

/* Same contract in float64 throughout (the float64 run of the reference's step). */
int ibis_step_f64(double* prog, const double* stat, const double* forc, double* diag, double* acc, int ncell,
                  int ld, int nstep, const IbisParams* params, int* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IBIS_B200_H */
