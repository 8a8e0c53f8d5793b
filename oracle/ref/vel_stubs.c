/*
 * vel_stubs.c -- link stubs for the functions model/hd/momentum/vel3d.c
 * calls outside the transport-mode preamble (momentum advection, open
 * boundaries, forcing, diagnostics).  TEST INFRASTRUCTURE ONLY: the preamble
 * the checker runs (set_dz_at_u1/u2, set_flux_3d, vel_w_update with a linear
 * free surface and no open boundaries) calls none of them, except
 * set_lateral_bc_eta, which only fills the elevation's lateral ghosts for the
 * non-linear surface terms (vel3d.c:5209-5212) and is a no-op here.
 */
/* (no SHOC header: the stubs below only give the linker each symbol) */

void set_lateral_bc_eta(double *eta, int nbpt, int *bpt, int *bin, int *bin2, int mode) {
  (void)eta; (void)nbpt; (void)bpt; (void)bin; (void)bin2; (void)mode;
}
/* never called on the preamble's path */
void advect_u1_3d(void) {}
void advect_u1_3d_ang_flux_b(void) {}
void advect_u2_3d(void) {}
void advect_u2_3d_ang_flux_b(void) {}
void bdry_closure(void) {}
void bdry_eval_tr_m(void) {}
void bdry_eval_tr_w(void) {}
void bdry_eval_u1_m(void) {}
void bdry_eval_u1_w(void) {}
void bdry_eval_u2_m(void) {}
void bdry_eval_u2_w(void) {}
void bdry_reconfigure(void) {}
void bdry_transfer_u1(void) {}
void bdry_transfer_u2(void) {}
void calc_cfl(void) {}
void calc_heatf(void) {}
void calc_saltf(void) {}
void check_flux(void) {}
void do_vel_relax(void) {}
void dp_vel3d_post_p1(void) {}
void dp_vel3d_post_p2(void) {}
void dp_vel3d_step_p1(void) {}
void dp_vel3d_step_p2(void) {}
void ekman_pump_e1(void) {}
void ekman_pump_e2(void) {}
void emstag(void) {}
void get_local_sur(void) {}
void global_interp_e1(void) {}
void global_interp_e2(void) {}
void global_interp_post(void) {}
void global_interp_pre(void) {}
void init_sigma(void) {}
void interp_adjust_e1(void) {}
void interp_adjust_e2(void) {}
void interp_dz_at_u1(void) {}
void interp_dz_at_u2(void) {}
void master_alert_fill(void) {}
void mdxbs(void) {}
void mdxns(void) {}
void mdybs(void) {}
void mdyns(void) {}
void reset_means_m(void) {}
void set_OBC(void) {}
void set_map_e1(void) {}
void set_map_e2(void) {}
void sourcesink_reinit(void) {}
void ss_momentum(void) {}
void ss_water(void) {}
void timeseries_init_w(void) {}
void vel2D_lbc(void) {}
