/*
 * Drop-in replacement for GAMERA-OP's step driver, src/solver_solve.c:23-536.
 *
 * Built inside a GAMERA-OP source tree in place of solver_solve.c (and of
 * boundary_conditions.c, replaced by gop_bc_record.c), it keeps the
 * reference's whole host side -- main (src/main.c), config.yaml, problem
 * hooks, geometry and weights, HDF5 output -- and moves the time loop onto
 * the GPU through the C ABI of include/gamera_op.h.  The state stays on the
 * device, which steps on its own up to the next host event (a dump time, a
 * log time or time_stop); at every output time (and once at the end)
 * the 18 store slots of gas[0] and gem are copied back into the host arrays
 * and written by the reference's own dump_data_hdf5 (src/hdf5_io.c:353-523),
 * so the per-step files keep their layout.
 *
 * Supported: one domain (proc_dims 1x1x1), COORD_TYPE 0 or 2, the BC library
 * of src/boundary_conditions.c, a background field B0 (the arrays main's
 * set_background_field leaves in gem go to the device), the spherical pole
 * ring average (doRingAverage = 1, with the pole fills of
 * spherical_boundary.c), no gravity.
 * GOP_PRECISION=mixed in the environment selects the mixed-precision stages.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <mpi.h>

#include "common.h"
#include "config.h"
#include "curvilinear.h"
#include "log.h"
#include "problem.h"
#include "setup_mpi.h"
#include "solver.h"
#include "utils.h"

#include "gamera_op.h"

extern char gop_gas_bc[6];
extern char gop_gem_bc[6];
void gop_bc_record_begin(void);

/* copy the device state into the reference's store slots */
static int download_store(gop_instance *h, int history) {
  size_t n3 = (size_t)config.NI * config.NJ * config.NK;
  double *gs = &gas[0][0][0][0][0];
  double *gm = &gem[0][0][0][0];
  return gop_download(h, gs, gm, history ? gs + (gas_rho_h - gas_rho) * n3 : NULL,
                      history ? gs + (gas_rho_p - gas_rho) * n3 : NULL,
                      history ? gm + (mag_bi_h - mag_bi) * n3 : NULL,
                      history ? gm + (mag_bi_p - mag_bi) * n3 : NULL,
                      gm + (mags_b1 - mag_bi) * n3,
                      history ? gm + (mags_b1_h - mag_bi) * n3 : NULL,
                      history ? gm + (mags_b1_p - mag_bi) * n3 : NULL);
}

static int gop_fail(gop_instance *h, const char *what, int rc) {
  log_error("gop solve(): %s failed (%d): %s", what, rc, gop_last_error());
  if (h) gop_destroy(h);
  return -1;
}

int solve(int nt) {
  if (config.proc_dims[0] * config.proc_dims[1] * config.proc_dims[2] != 1) {
    log_error("gop solve(): one domain per GPU instance (proc_dims 1 1 1)");
    return -1;
  }
  /* the boundary hook records its fills instead of applying them */
  gop_bc_record_begin();
  boundary_conditions();

  gop_desc d;
  memset(&d, 0, sizeof(d));
  d.ni = config.ni;
  d.nj = config.nj;
  d.nk = config.nk;
  /* H2 = r in spherical coordinates, 1 in Cartesian ones */
  d.coord = H2(2.0, 0.5, 0.0) == 2.0 ? GOP_COORD_SPHERICAL : GOP_COORD_CARTESIAN;
  double *xs[3];
  int N[3] = {config.NI, config.NJ, config.NK};
  for (int a = 0; a < 3; a++) xs[a] = (double *)malloc(sizeof(double) * N[a]);
  for (int i = 0; i < N[0]; i++) xs[0][i] = x1[i][0][0];
  for (int j = 0; j < N[1]; j++) xs[1][j] = x2[0][j][0];
  for (int k = 0; k < N[2]; k++) xs[2][k] = x3[0][0][k];
  d.x1 = xs[0];
  d.x2 = xs[1];
  d.x3 = xs[2];
  int periodic[3] = {problem_config.Boundary_i == BC_PERIODIC,
                     problem_config.Boundary_j == BC_PERIODIC,
                     problem_config.Boundary_k == BC_PERIODIC};
  for (int f = 0; f < 6; f++) {
    d.bc[f] = periodic[f / 2] ? 'p' : gop_gas_bc[f];
    d.gem_bc[f] = periodic[f / 2] ? 'p' : gop_gem_bc[f];
  }
  const char *prec = getenv("GOP_PRECISION");
  d.precision = (prec && strcmp(prec, "mixed") == 0) ? GOP_PREC_MIXED : GOP_PREC_FP64;
  d.gamma = gamma_val;
  d.cfl = CFL;
  d.ca = CA;
  d.rho_floor = rho_floor;
  d.p_floor = p_floor;
  d.ring_average = doRingAverage == 1;

  gop_instance *h = NULL;
  int rc = gop_create(&d, &h);
  for (int a = 0; a < 3; a++) free(xs[a]);
  if (rc) return gop_fail(NULL, "gop_create", rc);
  size_t n3 = (size_t)config.NI * config.NJ * config.NK;
  double *gs = &gas[0][0][0][0][0];
  double *gm = &gem[0][0][0][0];
  rc = gop_upload(h, gs, gm, read_restart ? gs + (gas_rho_p - gas_rho) * n3 : NULL,
                  read_restart ? gm + (mag_bi_p - mag_bi) * n3 : NULL, time_sim, dt0);
  if (rc) return gop_fail(h, "gop_upload", rc);
  if (B10 != Field_Default || B20 != Field_Default || B30 != Field_Default) {
    /* the background field set_background_field integrated on the host
     * (src/main.c:63): cell B0, its Lorentz force and the edge averages are
     * consecutive slots; the face averages b1..b3 are gathered per axis */
    double *face = (double *)malloc(9 * n3 * sizeof(double));
    if (!face) return gop_fail(h, "background staging", GOP_ENOMEM);
    const int fslot[3] = {B0AfaceI_b1, B0AfaceJ_b1, B0AfaceK_b1};
    for (int a = 0; a < 3; a++)
      memcpy(face + 3 * a * n3, gm + (fslot[a] - mag_bi) * n3, 3 * n3 * sizeof(double));
    rc = gop_set_background(h, gm + (B0_b1 - mag_bi) * n3, gm + (dmagsf_G_x1dir - mag_bi) * n3,
                            face, gm + (B0AedgeI_b1 - mag_bi) * n3);
    free(face);
    if (rc) return gop_fail(h, "gop_set_background", rc);
  }
  /* halo, boundary fill, derived variables and (fresh start) the AB2
   * history and initial dt0 (src/solver_solve.c:25-99) */
  rc = gop_prepare(h, read_restart ? 1 : 0);
  if (rc) return gop_fail(h, "gop_prepare", rc);
  if ((rc = download_store(h, 0))) return gop_fail(h, "gop_download", rc);
  gop_stats st;
  gop_get_stats(h, &st);
  divB_max = st.divb_max;

  double last_dump_time = time_sim;
  if (!read_restart) {
    log_info("Dump the initial state.");
    hdf_seq_num = -1;
    log_seq_num = 0;
    dump_data_hdf5(BASE_DAT_NAME);
    dump_extra_data(BASE_EXT_NAME);
    last_dump_time = 0;
  }
  dt0 = st.dt0;

  time_sim_start = time_sim;
  /* The reference needs the host only when time_sim reaches a dump or a log
   * threshold or passes time_stop (src/solver_solve.c:508-525).  So the
   * device steps on its own up to the first such event: gop_step stops after
   * the first step that takes time past its limit, and a limit just below a
   * threshold (nextafter) stops it at the first step reaching it, where the
   * host then acts exactly as the reference does after that step. */
  int n = 0;
  while (n < nt) {
    double stop = time_stop;
    const double t_dump = output_interval * (hdf_seq_num + 1);
    const double t_log = 0.1 * output_interval * (log_seq_num);
    if (nextafter(t_dump, -INFINITY) < stop) stop = nextafter(t_dump, -INFINITY);
    if (nextafter(t_log, -INFINITY) < stop) stop = nextafter(t_log, -INFINITY);
    /* an event already due (time_sim past the limit: the step counter's
     * first log, or a threshold the last step crossed twice over) happens
     * after the very next step */
    const int due = time_sim > stop;
    double t = 0.0;
    const int64_t before = st.steps;
    rc = gop_step(h, due ? 1 : nt - n, due ? 1e300 : stop, &t);
    if (rc) return gop_fail(h, "gop_step", rc);
    gop_get_stats(h, &st);
    if (st.steps == before) break; /* the limit was already behind: nothing ran */
    n += (int)(st.steps - before);
    time_sim = t;
    dt = st.dt;
    dt0 = st.dt0;
    divB_max = st.divb_max;
    if (dtout < dt)
      log_error("Rank=%d, Something wrong with dt, dt may be too large. dtout=%lf, dt=%lf\n", rank,
                dtout, dt);
    if (time_sim >= output_interval * (hdf_seq_num + 1)) {
      if ((rc = download_store(h, 1))) return gop_fail(h, "gop_download", rc);
      dump_data_hdf5(BASE_DAT_NAME);
      log_info("Output data at time %.15f\n", time_sim);
      last_dump_time = time_sim;
    }
    if (time_sim >= 0.1 * output_interval * (log_seq_num)) {
      log_info("Status at step %d: rank %d, Time %.15f, dt %.15f, max_divB for this rank is %.4e\n",
               n, rank, time_sim, dt, divB_max);
      log_seq_num = log_seq_num + 1;
    }
    if (time_sim > time_stop) {
      log_info("Step %d, Time %f, dt %f\n", n, time_sim, dt);
      log_info("This is the end\n");
      break;
    }
  }
  if (last_dump_time != time_sim) {
    if ((rc = download_store(h, 1))) return gop_fail(h, "gop_download", rc);
    dump_data_hdf5(BASE_DAT_NAME);
  }
  gop_destroy(h);
  return 0;
}
