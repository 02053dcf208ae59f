/* Generated from ibis_b200/layout.py by header_text(); do not edit by hand.
 *
 * Plane indices of the structure-of-arrays buffers of the hourly step.
 * Element (plane p, cell i) of a buffer with leading dimension ld lives at
 * buf[p * ld + i].  Forcing for a run of nstep hours is nstep consecutive
 * FORC blocks: step s, plane p, cell i at forc[(s * IBIS_FORC_COUNT + p) * ld + i].
 * The ACC buffer holds IBIS_ACC_COUNT value planes followed by the same
 * number of Kahan compensation planes.
 */
#ifndef IBIS_LAYOUT_H
#define IBIS_LAYOUT_H

/* PROG */
enum {
    IBIS_PROG_TSOI = 0,  /* soil.tsoi, 6 planes */
    IBIS_PROG_WSOI = 6,  /* soil.wsoi, 6 planes */
    IBIS_PROG_WISOI = 12,  /* soil.wisoi, 6 planes */
    IBIS_PROG_TG = 18,  /* soil.tg */
    IBIS_PROG_WPUD = 19,  /* soil.wpud */
    IBIS_PROG_WIPUD = 20,  /* soil.wipud */
    IBIS_PROG_TSOI_DEEP = 21,  /* soil.tsoi_deep, 3 planes */
    IBIS_PROG_FI = 24,  /* snow.fi */
    IBIS_PROG_TSNO = 25,  /* snow.tsno, 3 planes */
    IBIS_PROG_HSNO = 28,  /* snow.hsno, 3 planes */
    IBIS_PROG_TI = 31,  /* snow.ti */
    IBIS_PROG_TLSUB = 32,  /* snow.tlsub */
    IBIS_PROG_TU = 33,  /* canopy.tu */
    IBIS_PROG_TS = 34,  /* canopy.ts */
    IBIS_PROG_TL = 35,  /* canopy.tl */
    IBIS_PROG_T12 = 36,  /* canopy.t12 */
    IBIS_PROG_T34 = 37,  /* canopy.t34 */
    IBIS_PROG_Q12 = 38,  /* canopy.q12 */
    IBIS_PROG_Q34 = 39,  /* canopy.q34 */
    IBIS_PROG_WLIQU = 40,  /* canopy.wliqu */
    IBIS_PROG_WLIQS = 41,  /* canopy.wliqs */
    IBIS_PROG_WLIQL = 42,  /* canopy.wliql */
    IBIS_PROG_WSNOU = 43,  /* canopy.wsnou */
    IBIS_PROG_WSNOS = 44,  /* canopy.wsnos */
    IBIS_PROG_WSNOL = 45,  /* canopy.wsnol */
    IBIS_PROG_CI_UPPER = 46,  /* canopy.ci_upper, 2 planes */
    IBIS_PROG_GS_UPPER = 48,  /* canopy.gs_upper, 2 planes */
    IBIS_PROG_CS_UPPER = 50,  /* canopy.cs_upper, 2 planes */
    IBIS_PROG_CI_LOWER = 52,  /* canopy.ci_lower, 3 planes */
    IBIS_PROG_GS_LOWER = 55,  /* canopy.gs_lower, 3 planes */
    IBIS_PROG_CS_LOWER = 58,  /* canopy.cs_lower, 3 planes */
    IBIS_PROG_A10SCALPARAMU = 61,  /* canopy.a10scalparamu */
    IBIS_PROG_A10DAYLIGHTU = 62,  /* canopy.a10daylightu */
    IBIS_PROG_A10SCALPARAML = 63,  /* canopy.a10scalparaml */
    IBIS_PROG_A10DAYLIGHTL = 64,  /* canopy.a10daylightl */
    IBIS_PROG_FIREFAC = 65,  /* vegetation.firefac */
    IBIS_PROG_NYTIMES = 66,  /* vegetation.nytimes */
    IBIS_PROG_NFIRESTEP = 67,  /* vegetation.nfirestep */
    IBIS_PROG_SDRY = 68,  /* vegetation.sdry */
    IBIS_PROG_NFIRESTEP_VPD = 69,  /* vegetation.nfirestep_vpd */
    IBIS_PROG_SDRY_VPD = 70,  /* vegetation.sdry_vpd */
    IBIS_PROG_COUNT = 71
};

/* STAT */
enum {
    IBIS_STAT_POROS = 0,  /* soil.poros, 6 planes */
    IBIS_STAT_HYDRAUL = 6,  /* soil.hydraul, 6 planes */
    IBIS_STAT_SUCTION = 12,  /* soil.suction, 6 planes */
    IBIS_STAT_BEX = 18,  /* soil.bex, 6 planes */
    IBIS_STAT_SFIELD = 24,  /* soil.sfield, 6 planes */
    IBIS_STAT_SWILT = 30,  /* soil.swilt, 6 planes */
    IBIS_STAT_SAND = 36,  /* soil.sand, 6 planes */
    IBIS_STAT_CLAY = 42,  /* soil.clay, 6 planes */
    IBIS_STAT_CSOI = 48,  /* soil.csoi, 6 planes */
    IBIS_STAT_RHOSOI = 54,  /* soil.rhosoi, 6 planes */
    IBIS_STAT_ALBSAV = 60,  /* soil.albsav */
    IBIS_STAT_ALBSAN = 61,  /* soil.albsan */
    IBIS_STAT_Z0SOI = 62,  /* soil.z0soi */
    IBIS_STAT_LAI = 63,  /* vegetation.lai, 2 planes */
    IBIS_STAT_SAI = 65,  /* vegetation.sai, 2 planes */
    IBIS_STAT_ZTOP = 67,  /* vegetation.ztop, 2 planes */
    IBIS_STAT_ZBOT = 69,  /* vegetation.zbot, 2 planes */
    IBIS_STAT_FU = 71,  /* vegetation.fu */
    IBIS_STAT_FL = 72,  /* vegetation.fl */
    IBIS_STAT_FRAC = 73,  /* vegetation.frac, 12 planes */
    IBIS_STAT_EXIST = 85,  /* vegetation.exist, 12 planes */
    IBIS_STAT_CBIOW = 97,  /* vegetation.cbiow, 12 planes */
    IBIS_STAT_CBIOR = 109,  /* vegetation.cbior, 12 planes */
    IBIS_STAT_SAPFRAC = 121,  /* vegetation.sapfrac */
    IBIS_STAT_TCO2MIC = 122,  /* vegetation.tco2mic */
    IBIS_STAT_F_INUND = 123,  /* methane.f_inund */
    IBIS_STAT_ZWT_OBS = 124,  /* methane.zwt_obs */
    IBIS_STAT_ACCLIM_X = 125,  /* seasonal.acclim_x */
    IBIS_STAT_TD = 126,  /* atm.td */
    IBIS_STAT_CROPFRAC = 127,  /* sim.cropfrac */
    IBIS_STAT_FORGANIC = 128,  /* sim.forganic, 6 planes */
    IBIS_STAT_CH4_BAND = 134,  /* sim.ch4_band */
    IBIS_STAT_COUNT = 135
};

/* FORC */
enum {
    IBIS_FORC_TA = 0,  /* atm.ta */
    IBIS_FORC_QA = 1,  /* atm.qa */
    IBIS_FORC_UA = 2,  /* atm.ua */
    IBIS_FORC_PSURF = 3,  /* atm.psurf */
    IBIS_FORC_COSZEN = 4,  /* atm.coszen */
    IBIS_FORC_SOLAD = 5,  /* atm.solad, 2 planes */
    IBIS_FORC_SOLAI = 7,  /* atm.solai, 2 planes */
    IBIS_FORC_FIRA = 9,  /* atm.fira */
    IBIS_FORC_RAINA = 10,  /* atm.raina */
    IBIS_FORC_SNOWA = 11,  /* atm.snowa */
    IBIS_FORC_COUNT = 12
};

/* DIAG */
enum {
    IBIS_DIAG_AN_UPPER = 0,  /* canopy.an_upper, 2 planes */
    IBIS_DIAG_AG_UPPER = 2,  /* canopy.ag_upper, 2 planes */
    IBIS_DIAG_AN_LOWER = 4,  /* canopy.an_lower, 3 planes */
    IBIS_DIAG_AG_LOWER = 7,  /* canopy.ag_lower, 3 planes */
    IBIS_DIAG_FWETU = 10,  /* canopy.fwetu */
    IBIS_DIAG_FWETS = 11,  /* canopy.fwets */
    IBIS_DIAG_FWETL = 12,  /* canopy.fwetl */
    IBIS_DIAG_RLIQU = 13,  /* canopy.rliqu */
    IBIS_DIAG_RLIQS = 14,  /* canopy.rliqs */
    IBIS_DIAG_RLIQL = 15,  /* canopy.rliql */
    IBIS_DIAG_SOLU = 16,  /* canopy.solu */
    IBIS_DIAG_SOLS = 17,  /* canopy.sols */
    IBIS_DIAG_SOLL = 18,  /* canopy.soll */
    IBIS_DIAG_SOLG = 19,  /* canopy.solg */
    IBIS_DIAG_SOLI = 20,  /* canopy.soli */
    IBIS_DIAG_FIRU = 21,  /* canopy.firu */
    IBIS_DIAG_FIRS = 22,  /* canopy.firs */
    IBIS_DIAG_FIRL = 23,  /* canopy.firl */
    IBIS_DIAG_FIRG = 24,  /* canopy.firg */
    IBIS_DIAG_FIRI = 25,  /* canopy.firi */
    IBIS_DIAG_FIRB = 26,  /* canopy.firb */
    IBIS_DIAG_ASURD = 27,  /* canopy.asurd, 2 planes */
    IBIS_DIAG_ASURI = 29,  /* canopy.asuri, 2 planes */
    IBIS_DIAG_TOPPARU = 31,  /* canopy.topparu */
    IBIS_DIAG_TOPPARL = 32,  /* canopy.topparl */
    IBIS_DIAG_SCALCOEFU = 33,  /* canopy.scalcoefu, 4 planes */
    IBIS_DIAG_SCALCOEFL = 37,  /* canopy.scalcoefl, 4 planes */
    IBIS_DIAG_FSENU = 41,  /* canopy.fsenu */
    IBIS_DIAG_FSENS = 42,  /* canopy.fsens */
    IBIS_DIAG_FSENL = 43,  /* canopy.fsenl */
    IBIS_DIAG_FSENG = 44,  /* canopy.fseng */
    IBIS_DIAG_FSENI = 45,  /* canopy.fseni */
    IBIS_DIAG_FVAPG = 46,  /* canopy.fvapg */
    IBIS_DIAG_FVAPI = 47,  /* canopy.fvapi */
    IBIS_DIAG_RAING = 48,  /* canopy.raing */
    IBIS_DIAG_SNOWG = 49,  /* canopy.snowg */
    IBIS_DIAG_RHOA = 50,  /* canopy.rhoa */
    IBIS_DIAG_CONSOI = 51,  /* soil.consoi, 6 planes */
    IBIS_DIAG_HFLO = 57,  /* soil.hflo, 7 planes */
    IBIS_DIAG_HEATG = 64,  /* soil.heatg */
    IBIS_DIAG_HVASUG = 65,  /* soil.hvasug */
    IBIS_DIAG_QGLIF = 66,  /* soil.qglif, 4 planes */
    IBIS_DIAG_STRESSTU = 70,  /* soil.stresstu */
    IBIS_DIAG_STRESSTL = 71,  /* soil.stresstl */
    IBIS_DIAG_STRESSU = 72,  /* soil.stressu, 6 planes */
    IBIS_DIAG_STRESSL = 78,  /* soil.stressl, 6 planes */
    IBIS_DIAG_POROSFLO = 84,  /* soil.porosflo, 6 planes */
    IBIS_DIAG_HEATI = 90,  /* snow.heati */
    IBIS_DIAG_HVASUI = 91,  /* snow.hvasui */
    IBIS_DIAG_GINVAP = 92,  /* hydrology.ginvap */
    IBIS_DIAG_GSUVAP = 93,  /* hydrology.gsuvap */
    IBIS_DIAG_GTRANS = 94,  /* hydrology.gtrans */
    IBIS_DIAG_GTRANSU = 95,  /* hydrology.gtransu */
    IBIS_DIAG_GTRANSL = 96,  /* hydrology.gtransl */
    IBIS_DIAG_GRUNOF = 97,  /* hydrology.grunof */
    IBIS_DIAG_GDRAIN = 98,  /* hydrology.gdrain */
    IBIS_DIAG_GADJUST = 99,  /* hydrology.gadjust */
    IBIS_DIAG_WTOT = 100,  /* hydrology.wtot */
    IBIS_DIAG_RAING_AVG = 101,  /* hydrology.raing_avg */
    IBIS_DIAG_TRAING_AVG = 102,  /* hydrology.traing_avg */
    IBIS_DIAG_FHTOP_SOIL = 103,  /* hydrology.fhtop_soil */
    IBIS_DIAG_RAINL = 104,  /* hydrology.rainl */
    IBIS_DIAG_SNOWL = 105,  /* hydrology.snowl */
    IBIS_DIAG_TRAINL = 106,  /* hydrology.trainl */
    IBIS_DIAG_TSNOWL = 107,  /* hydrology.tsnowl */
    IBIS_DIAG_SFLO_BOT = 108,  /* hydrology.sflo_bot */
    IBIS_DIAG_FHTOP_SNOW = 109,  /* hydrology.fhtop_snow */
    IBIS_DIAG_FSENA = 110,  /* canopy.fsena */
    IBIS_DIAG_COUNT = 111
};

/* ACC */
enum {
    IBIS_ACC_ADRAIN = 0,  /* summary.adrain */
    IBIS_ACC_ADSNOW = 1,  /* summary.adsnow */
    IBIS_ACC_ADAET = 2,  /* summary.adaet */
    IBIS_ACC_A10ANCUB = 3,  /* summary.a10ancub */
    IBIS_ACC_A10ANCLS = 4,  /* summary.a10ancls */
    IBIS_ACC_A10ANCL3 = 5,  /* summary.a10ancl3 */
    IBIS_ACC_A10ANCL4 = 6,  /* summary.a10ancl4 */
    IBIS_ACC_AYNPP = 7,  /* summary.aynpp, 12 planes */
    IBIS_ACC_AYNPPTOT = 19,  /* summary.aynpptot */
    IBIS_ACC_AYGPPTOT = 20,  /* summary.aygpptot */
    IBIS_ACC_AYTRUNOF = 21,  /* summary.aytrunof */
    IBIS_ACC_AYTDRAIN = 22,  /* summary.aytdrain */
    IBIS_ACC_CH4 = 23,  /* acc.ch4_day */
    IBIS_ACC_TSOI_MEAN = 24,  /* acc.tsoi_day, 6 planes */
    IBIS_ACC_WSOI_MEAN = 30,  /* acc.wsoi_day, 6 planes */
    IBIS_ACC_WISOI_MEAN = 36,  /* acc.wisoi_day, 6 planes */
    IBIS_ACC_TG_MEAN = 42,  /* acc.tg_day */
    IBIS_ACC_AFSENA = 43,  /* acc.fsena */
    IBIS_ACC_STRESSTU_LAST = 44,  /* soil.stresstu */
    IBIS_ACC_STRESSTL_LAST = 45,  /* soil.stresstl */
    IBIS_ACC_ET_TRANS = 46,  /* etparts.trans */
    IBIS_ACC_ET_INTERC = 47,  /* etparts.interc */
    IBIS_ACC_ET_SOILEV = 48,  /* etparts.soilev */
    IBIS_ACC_ET_SNOWSUB = 49,  /* etparts.snowsub */
    IBIS_ACC_NEE_NIGHT = 50,  /* neeparts.night */
    IBIS_ACC_NEE_DAY = 51,  /* neeparts.day */
    IBIS_ACC_COUNT = 52
};

/* RUN */
enum {
    IBIS_RUN_VMAX = 0,  /* stomata_params.vmax_pft, 12 planes */
    IBIS_RUN_COEFM = 12,  /* stomata_params.coefm, 5 planes */
    IBIS_RUN_STRESSFAC = 17,  /* stomata_params.stressfac */
    IBIS_RUN_SOIL_BETA_POWER = 18,  /* canopy.soil_beta_power */
    IBIS_RUN_WLIQUMAX = 19,  /* interception.wliqumax */
    IBIS_RUN_WLIQSMAX = 20,  /* interception.wliqsmax */
    IBIS_RUN_WLIQLMAX = 21,  /* interception.wliqlmax */
    IBIS_RUN_FMAX = 22,  /* interception.fmax */
    IBIS_RUN_R_CH4 = 23,  /* methane.r_ch4 */
    IBIS_RUN_Q10P = 24,  /* methane.q10p */
    IBIS_RUN_Z_TAU = 25,  /* methane.z_tau */
    IBIS_RUN_TAU_OXID = 26,  /* methane.tau_oxid */
    IBIS_RUN_Z_WT_MAX = 27,  /* methane.z_wt_max */
    IBIS_RUN_RWOOD = 28,  /* bgc_params.rwood */
    IBIS_RUN_RROOT = 29,  /* bgc_params.rroot */
    IBIS_RUN_RGROWTH = 30,  /* bgc_params.rgrowth */
    IBIS_RUN_COUNT = 31
};

/* YEARLY */
enum {
    IBIS_YEARLY_AYGPPTOT = 0,  /* summary.aygpptot */
    IBIS_YEARLY_AYNPPTOT = 1,  /* summary.aynpptot */
    IBIS_YEARLY_ADAET = 2,  /* summary.adaet */
    IBIS_YEARLY_AFSENA = 3,  /* acc.fsena */
    IBIS_YEARLY_AYTRUNOF = 4,  /* summary.aytrunof */
    IBIS_YEARLY_AYTDRAIN = 5,  /* summary.aytdrain */
    IBIS_YEARLY_CH4 = 6,  /* acc.ch4_day */
    IBIS_YEARLY_COUNT = 7
};

/* DAILY */
enum {
    IBIS_DAILY_TD = 0,  /* daily_weather.td */
    IBIS_DAILY_TMAX = 1,  /* daily_weather.tmax */
    IBIS_DAILY_TMIN = 2,  /* daily_weather.tmin */
    IBIS_DAILY_CLOUD = 3,  /* daily_weather.cloud */
    IBIS_DAILY_PRECIP = 4,  /* daily_weather.precip */
    IBIS_DAILY_PSURF = 5,  /* daily_weather.psurf */
    IBIS_DAILY_QD = 6,  /* daily_weather.qd */
    IBIS_DAILY_UD = 7,  /* daily_weather.ud */
    IBIS_DAILY_FIRA = 8,  /* gswp3.rlds */
    IBIS_DAILY_COUNT = 9
};

/* DAYST */
enum {
    IBIS_DAYST_PLAI = 0,  /* vegetation.plai, 12 planes */
    IBIS_DAYST_TC = 12,  /* vegetation.tc */
    IBIS_DAYST_TEMPU = 13,  /* vegetation.tempu */
    IBIS_DAYST_TEMPL = 14,  /* vegetation.templ */
    IBIS_DAYST_AGDDU = 15,  /* vegetation.agddu */
    IBIS_DAYST_AGDDL = 16,  /* vegetation.agddl */
    IBIS_DAYST_DROPU = 17,  /* vegetation.dropu */
    IBIS_DAYST_DROPLS = 18,  /* vegetation.dropls */
    IBIS_DAYST_DROPL3 = 19,  /* vegetation.dropl3 */
    IBIS_DAYST_DROPL4 = 20,  /* vegetation.dropl4 */
    IBIS_DAYST_TCO2ROOT = 21,  /* vegetation.tco2root */
    IBIS_DAYST_TNMIN = 22,  /* vegetation.tnmin */
    IBIS_DAYST_A10TD = 23,  /* summary.a10td */
    IBIS_DAYST_A10ANCUB = 24,  /* summary.a10ancub */
    IBIS_DAYST_A10ANCLS = 25,  /* summary.a10ancls */
    IBIS_DAYST_A10ANCL3 = 26,  /* summary.a10ancl3 */
    IBIS_DAYST_A10ANCL4 = 27,  /* summary.a10ancl4 */
    IBIS_DAYST_AYPRCP = 28,  /* summary.ayprcp */
    IBIS_DAYST_AYAET = 29,  /* summary.ayaet */
    IBIS_DAYST_AYCO2MIC = 30,  /* summary.ayco2mic */
    IBIS_DAYST_AYCO2ROOT = 31,  /* summary.ayco2root */
    IBIS_DAYST_STOREDN = 32,  /* summary.storedn */
    IBIS_DAYST_YRLEACH = 33,  /* summary.yrleach */
    IBIS_DAYST_YNLEACH = 34,  /* summary.ynleach */
    IBIS_DAYST_CLITLM = 35,  /* carbon.clitlm */
    IBIS_DAYST_CLITLS = 36,  /* carbon.clitls */
    IBIS_DAYST_CLITLL = 37,  /* carbon.clitll */
    IBIS_DAYST_CLITRM = 38,  /* carbon.clitrm */
    IBIS_DAYST_CLITRS = 39,  /* carbon.clitrs */
    IBIS_DAYST_CLITRL = 40,  /* carbon.clitrl */
    IBIS_DAYST_CLITWM = 41,  /* carbon.clitwm */
    IBIS_DAYST_CLITWS = 42,  /* carbon.clitws */
    IBIS_DAYST_CLITWL = 43,  /* carbon.clitwl */
    IBIS_DAYST_CSOISLOP = 44,  /* carbon.csoislop */
    IBIS_DAYST_CSOISLON = 45,  /* carbon.csoislon */
    IBIS_DAYST_CSOIPAS = 46,  /* carbon.csoipas */
    IBIS_DAYST_TOTCMIC = 47,  /* carbon.totcmic */
    IBIS_DAYST_DECOMPL = 48,  /* carbon.decompl */
    IBIS_DAYST_DECOMPS = 49,  /* carbon.decomps */
    IBIS_DAYST_TOTLIT = 50,  /* carbon.totlit */
    IBIS_DAYST_TOTALIT = 51,  /* carbon.totalit */
    IBIS_DAYST_TOTRLIT = 52,  /* carbon.totrlit */
    IBIS_DAYST_TOTCSOI = 53,  /* carbon.totcsoi */
    IBIS_DAYST_TOTFALL = 54,  /* carbon.totfall */
    IBIS_DAYST_FALLL = 55,  /* carbon.falll */
    IBIS_DAYST_FALLR = 56,  /* carbon.fallr */
    IBIS_DAYST_FALLW = 57,  /* carbon.fallw */
    IBIS_DAYST_ACCLIM_X = 58,  /* seasonal.acclim_x */
    IBIS_DAYST_SSEN_U = 59,  /* seasonal.ssen_u */
    IBIS_DAYST_SSEN_L = 60,  /* seasonal.ssen_l */
    IBIS_DAYST_AYSTRESSU = 61,  /* stress.aystressu */
    IBIS_DAYST_AYSTRESSL = 62,  /* stress.aystressl */
    IBIS_DAYST_STRESS_NDAY = 63,  /* stress.nday */
    IBIS_DAYST_LATITUDE = 64,  /* params.latitude */
    IBIS_DAYST_COUNT = 65
};

/* WET */
enum {
    IBIS_WET_FLUX = 0,  /* wetland.flux */
    IBIS_WET_ANNUAL = 1,  /* wetland.annual */
    IBIS_WET_ZWT = 2,  /* wetland.zwt */
    IBIS_WET_RH0 = 3,  /* summary.ayco2mic */
    IBIS_WET_CH4C = 4,  /* summary.ayrh_ch4c */
    IBIS_WET_COUNT = 5
};

/* Parameter record of the hourly step (all double; passed by value). */
typedef struct IbisParams {
    double stef;
    double vonk;
    double grav;
    double tmelt;
    double hvap;
    double hfus;
    double hsub;
    double ch2o;
    double cice;
    double cair;
    double cvap;
    double rair;
    double rvap;
    double cappa;
    double rhow;
    double epsilon;
    double dtime;
    double co2conc;
    double z0sno;
    double rhos;
    double consno;
    double hsnotop;
    double hsnomin;
    double fimin;
    double fimax;
    double rhoveg[4];
    double tauveg[4];
    double oriev[2];
    double orieh[2];
    double omegasno[2];
    double cleaf;
    double cstem;
    double cgrass;
    double dleaf[2];
    double dstem[2];
    double alaiml;
    double alaimu;
    double chu;
    double chs;
    double chl;
    double soil_beta_power;
    double wliqumax;
    double wliqsmax;
    double wliqlmax;
    double wsnoumax;
    double wsnosmax;
    double wsnolmax;
    double tdripu;
    double tdrips;
    double tdripl;
    double tblowu;
    double tblows;
    double tblowl;
    double fmax;
    double tau15;
    double kc15;
    double ko15;
    double cimax;
    double o2conc;
    double alpha3;
    double theta3;
    double beta3;
    double alpha4;
    double theta4;
    double beta4;
    double gamma[5];
    double coefm[5];
    double coefb[5];
    double gsmin[5];
    double vmax_pft[12];
    double stressfac;
    double cap_kn;
    double coefm_pft[12];
    double acclim_mask[12];
    double acclim_s0_pft[12];
    double acclim_smax_pft[12];
    double frost_t0;
    double frost_t1;
    double crop_vmax_scale_c3;
    double crop_vmax_scale_c4;
    double crop_c4_share;
    double wpudmax;
    double zwpmax;
    double bperm;
    double rhosoi_val;
    double csoi_mineral_val;
    double hsoi[6];
    double froot[12];
    double hsoi_bed[3];
    double consoi_bed;
    double rhosoi_bed;
    double csoi_bed;
    double d_crit;
    double vpd_ref;
    double d_crit_vpd;
    double flux_max;
    double t_max_dev;
    double sat_crit;
    double z_max;
    double r_ch4;
    double q10p;
    double t_ref;
    double z_wt_max;
    double z_wt_ref;
    double z_tau;
    double tau_oxid;
    double ch4b_sat_crit[3];
    double ch4b_z_max[3];
    double ch4b_r_ch4[3];
    double ch4b_q10p[3];
    double ch4b_t_ref[3];
    double ch4b_z_wt_max[3];
    double ch4b_z_wt_ref[3];
    double ch4b_z_tau[3];
    double ch4b_tau_oxid[3];
    double rwood[12];
    double rroot[12];
    double rgrowth[12];
    double ndaypy;
    unsigned int flags;   /* IBIS_FLAG_* */
    unsigned int _pad;
} IbisParams;

/* X-macro over the record: S(name) for scalars, A(name, count) for tables. */
#define IBIS_PARAM_LIST(S, A) \
    S(stef) \
    S(vonk) \
    S(grav) \
    S(tmelt) \
    S(hvap) \
    S(hfus) \
    S(hsub) \
    S(ch2o) \
    S(cice) \
    S(cair) \
    S(cvap) \
    S(rair) \
    S(rvap) \
    S(cappa) \
    S(rhow) \
    S(epsilon) \
    S(dtime) \
    S(co2conc) \
    S(z0sno) \
    S(rhos) \
    S(consno) \
    S(hsnotop) \
    S(hsnomin) \
    S(fimin) \
    S(fimax) \
    A(rhoveg, 4) \
    A(tauveg, 4) \
    A(oriev, 2) \
    A(orieh, 2) \
    A(omegasno, 2) \
    S(cleaf) \
    S(cstem) \
    S(cgrass) \
    A(dleaf, 2) \
    A(dstem, 2) \
    S(alaiml) \
    S(alaimu) \
    S(chu) \
    S(chs) \
    S(chl) \
    S(soil_beta_power) \
    S(wliqumax) \
    S(wliqsmax) \
    S(wliqlmax) \
    S(wsnoumax) \
    S(wsnosmax) \
    S(wsnolmax) \
    S(tdripu) \
    S(tdrips) \
    S(tdripl) \
    S(tblowu) \
    S(tblows) \
    S(tblowl) \
    S(fmax) \
    S(tau15) \
    S(kc15) \
    S(ko15) \
    S(cimax) \
    S(o2conc) \
    S(alpha3) \
    S(theta3) \
    S(beta3) \
    S(alpha4) \
    S(theta4) \
    S(beta4) \
    A(gamma, 5) \
    A(coefm, 5) \
    A(coefb, 5) \
    A(gsmin, 5) \
    A(vmax_pft, 12) \
    S(stressfac) \
    S(cap_kn) \
    A(coefm_pft, 12) \
    A(acclim_mask, 12) \
    A(acclim_s0_pft, 12) \
    A(acclim_smax_pft, 12) \
    S(frost_t0) \
    S(frost_t1) \
    S(crop_vmax_scale_c3) \
    S(crop_vmax_scale_c4) \
    S(crop_c4_share) \
    S(wpudmax) \
    S(zwpmax) \
    S(bperm) \
    S(rhosoi_val) \
    S(csoi_mineral_val) \
    A(hsoi, 6) \
    A(froot, 12) \
    A(hsoi_bed, 3) \
    S(consoi_bed) \
    S(rhosoi_bed) \
    S(csoi_bed) \
    S(d_crit) \
    S(vpd_ref) \
    S(d_crit_vpd) \
    S(flux_max) \
    S(t_max_dev) \
    S(sat_crit) \
    S(z_max) \
    S(r_ch4) \
    S(q10p) \
    S(t_ref) \
    S(z_wt_max) \
    S(z_wt_ref) \
    S(z_tau) \
    S(tau_oxid) \
    A(ch4b_sat_crit, 3) \
    A(ch4b_z_max, 3) \
    A(ch4b_r_ch4, 3) \
    A(ch4b_q10p, 3) \
    A(ch4b_t_ref, 3) \
    A(ch4b_z_wt_max, 3) \
    A(ch4b_z_wt_ref, 3) \
    A(ch4b_z_tau, 3) \
    A(ch4b_tau_oxid, 3) \
    A(rwood, 12) \
    A(rroot, 12) \
    A(rgrowth, 12) \
    S(ndaypy) \


#define IBIS_FLAG_BEDROCK 1u
#define IBIS_FLAG_H2O_CONSISTENT 2u
#define IBIS_FLAG_SUNSHADE_U 4u
#define IBIS_FLAG_SUNSHADE_L 8u
#define IBIS_FLAG_ACC 16u
#define IBIS_FLAG_CH4 32u
#define IBIS_FLAG_SOIL_MEANS 64u
#define IBIS_FLAG_DIAG 128u
#define IBIS_FLAG_KAHAN 256u
#define IBIS_FLAG_ZWT_OBS 512u
#define IBIS_FLAG_ETPARTS 1024u
#define IBIS_FLAG_NEEPARTS 2048u
#define IBIS_FLAG_VMAX_MIX 4096u
#define IBIS_FLAG_COEFM_MIX 8192u
#define IBIS_FLAG_GPP_CAPACITY 16384u
#define IBIS_FLAG_ACCLIM 32768u
#define IBIS_FLAG_ACCLIM_LIGHT 65536u
#define IBIS_FLAG_FROST 131072u
#define IBIS_FLAG_CAP_SCALE_U 262144u
#define IBIS_FLAG_CAP_SCALE_L 524288u
#define IBIS_FLAG_LEAF_ONLY 1048576u
#define IBIS_FLAG_CROP 2097152u
#define IBIS_FLAG_FORGANIC 4194304u
#define IBIS_FLAG_CH4_BANDS 8388608u
#define IBIS_FLAGS_X3 8384512u   /* any of these selects the IBIS 3.0 kernels */

/* Parameters of the daily cadence (phenology, soil biogeochemistry), all double. */
typedef struct IbisDayParams {
    double ddays;
    double tthresh_u_offset;
    double tthresh_u_abs;
    double gthresh_u_c;
    double gdd_thresh_u;
    double gdd_ramp_u;
    double tthresh_l_c;
    double gthresh_l_c;
    double gdd_thresh_l;
    double gdd_ramp_l;
    double drop_thresh;
    double drop_stress_thresh;
    double drop_floor;
    double stress_accum_tmin;
    double sen_photoperiod_u;
    double sen_pstart_u;
    double sen_tb_u;
    double sen_ycrit_u;
    double sen_photoperiod_l;
    double sen_pstart_l;
    double sen_tb_l;
    double sen_ycrit_l;
    double lig_frac;
    double fbsom;
    double effac;
    double bgc_fmax;
    double rconst;
    double cnleaf;
    double cnroot;
    double cnwood;
    double cnr[8];
    double klm;
    double kls;
    double kll;
    double krm;
    double krs;
    double krl;
    double kwm;
    double kws;
    double kwl;
    double kbn;
    double kbp;
    double knb;
    double kns;
    double kpb;
    double kps;
    double ksb;
    double ylm;
    double yls;
    double yll;
    double yrm;
    double yrs;
    double yrl;
    double ywm;
    double yws;
    double ywl;
    double ybn;
    double ybp;
    double yps;
    double yns;
    double ysb;
    double ypb;
    double ynb;
    double lt_e0;
    double wfps_opt;
    double k_scale;
    double acclim_tau;
    double jday;
    double seasonal_on;
    double stress_on;
} IbisDayParams;

#endif /* IBIS_LAYOUT_H */
