/*
 * dsmsgt_host.h -- driver-side helpers of the SGT engine.
 *
 * These are the steps the reference's Fortran drivers perform before their
 * frequency loop: reading the parameter file from stdin (pinput,
 * src/SGTpsv/others.f90:1-72), DSM.config (readDSMconf, :74-111), the
 * polynomial model file (readpsvmodel, :114-129, and the read at
 * src/SGTpsv/SGTpsv-MPI.f90:100-105), building the radial grid and the
 * element integrals (SGTpsv-MPI.f90:214-477, SGTsh-MPI.f90:66-347).  They
 * fill the set-up structs of dsmsgt.h.  A Fortran driver would keep its
 * own code for these steps and only bind dsmsgt.h; the C++ drivers and the
 * test harness of this project use these helpers instead.
 *
 * All text arguments are the full contents of the respective files.
 */
#ifndef DSMSGT_HOST_H
#define DSMSGT_HOST_H

#include "dsmsgt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dsm_bundle dsm_bundle_t;   /* owns every array of a set-up */

/* Parsed parameter file (the 9 items of pinput). */
typedef struct dsm_params {
    char   dsmconf[256], outdir[256], model[256], modelname[128];
    double tlen, rmin_, rmax_, rdelta_, r0min;
    double thetamin, thetamax, thetadelta;
    int    imin, imax;
    int    rsgt_switch, tsgt_switch, synn_switch, psgt_switch;
} dsm_params_t;

int dsm_parse_params(const char *param_text, dsm_params_t *out);

/* SH: builds the set-up of SGTsh (outer core cut, grid, element
 * integrals).  The returned set-up points into the bundle. */
int dsm_sh_setup_build(const dsm_params_t *par, const char *conf_text,
                       const char *model_text, dsm_bundle_t **bundle,
                       const dsm_sh_setup_t **setup);

/* PSV: builds the set-up of SGTpsv. */
int dsm_psv_setup_build(const dsm_params_t *par, const char *conf_text,
                        const char *model_text, dsm_bundle_t **bundle,
                        const dsm_psv_setup_t **setup);

/* PSV with the element integrals (src/SGTpsv/SGTpsv-MPI.f90:383-477:
 * calmatc, pinteg, caltl, calhl, calt, calh5, submat, mtrnp, calhm1,
 * calhm2, mtrnp2) computed on CUDA device `device`, one thread per layer /
 * node column; the rest of the set-up as dsm_psv_setup_build, and the same
 * arrays bit for bit.  For requests that set up many models. */
int dsm_psv_setup_build_device(const dsm_params_t *par, const char *conf_text,
                               const char *model_text, int device, dsm_bundle_t **bundle,
                               const dsm_psv_setup_t **setup);

/* Number of radial nodes / unknowns of a bundle, for reports. */
int dsm_bundle_info(const dsm_bundle_t *bundle, int *n_nodes, int *n_unknowns);

void dsm_bundle_free(dsm_bundle_t *bundle);
const char *dsm_host_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
