/* CPU oracle for the waam_twin coupled melt-pool step -- TEST INFRASTRUCTURE.
 *
 * A plain-C (float32) restatement of the reference's Taichi kernels
 * (kernels.py, cumulant_kernel.py of THEDARKDEACON/waam_solver).  Only the
 * parity tests, the smoke check and the CPU-baseline leg of bench.py load it;
 * the product never links it.  Every function cites the reference kernel it
 * restates.  Layout matches the reference grid: scalar fields are (nx, ny, nz)
 * row-major with k fastest, populations are (19, nx, ny, nz); flags are int32
 * with FLUID=0, SOLID=1, GAS=2, IFACE=4.
 *
 * Semantics pinned where the reference is racy:
 *   wo_advect_diffuse_temperature  -- neighbour reads of H see the value from
 *                                     before the kernel (snapshot);
 *   wo_apply_contact_angle_phi_bc  -- sequential in k within a column,
 *                                     other columns read from the snapshot;
 *   wo_feed_wire_surface           -- serial lexicographic order;
 *   arc-weight and other sums      -- accumulated in double.
 */
#ifndef WAAM_ORACLE_H
#define WAAM_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

int wo_num_threads(void);
void wo_expf_array(const float* x, float* y, int64_t n);
void wo_set_num_threads(int n);

void wo_init_grid(float* f, float* rho, float* ux, float* uy, float* uz, float* T, float* H,
                  float* f_l, float* phi, int32_t* flags, int nx, int ny, int nz, float T_amb,
                  float rho0, float cp_rho, int nz_solid, int pi0, int pi1, int pj0, int pj1);
void wo_clear_forces(float* Fx, float* Fy, float* Fz, int64_t n);
double wo_inject_arc_heat(float* H, const int32_t* flags, const float* f_l, int nx, int ny, int nz,
                          float arc_i, float arc_j, float arc_k, float Q_w, float sigma, float dt,
                          float dx3, float eta, float pen, int enable);
double wo_inject_goldak_heat(float* H, const int32_t* flags, const float* f_l, int nx, int ny,
                             int nz, float arc_i, float arc_j, float arc_k, float Q_w, float dt,
                             float dx3, float eta, float sign, float ff, float fr, float a_f,
                             float a_r, float b, float c, float pen, int enable);
void wo_clamp_enthalpy_ceiling_scalar(float* H, const int32_t* flags, int64_t n, float cp_rho,
                                      float Ts, float Tl, float T_cap, float L_rho);
void wo_advect_diffuse_temperature(float* H, const float* T, const float* ux, const float* uy,
                                   const float* uz, const int32_t* flags, int nx, int ny, int nz,
                                   float alpha_lu, float dt, float cp_rho);
void wo_update_phase(const float* H, float* T, float* f_l, int64_t n, float cp_rho, float L_rho,
                     float Ts, float Tl);
void wo_update_T_max(const float* T, float* T_max, const int32_t* flags, int64_t n);
void wo_update_cooling_rate(const float* T, float* T_prev, float* dT_dt, const int32_t* flags,
                            int64_t n, float dt_phys);
void wo_apply_thermal_boundary_losses(float* H, const float* T, const int32_t* flags, int nx,
                                      int ny, int nz, float T_amb, float h_conv, float eps_rad,
                                      int conv, int rad, float dt, float dx, float sigma_sb);
void wo_clamp_enthalpy_floor_scalar(float* H, float cp_rho, const int32_t* flags, int64_t n,
                                    float T_floor);
void wo_advect_phi(float* phi_dst, const float* phi_src, const float* ux, const float* uy,
                   const float* uz, const int32_t* flags, int nx, int ny, int nz);
void wo_reinitialize_phi(float* phi, const int32_t* flags, int64_t n);
void wo_apply_contact_angle_phi_bc(float* phi, const int32_t* flags, int nx, int ny, int nz,
                                   float theta);
void wo_update_flags_from_phi(const float* phi, const float* f_l, int32_t* flags, int nx, int ny,
                              int nz, int nz_solid);
void wo_sync_phi_liquid_fraction(const float* phi, float* f_l, const int32_t* flags, int64_t n);
void wo_compute_csf_tension(const float* phi, const int32_t* flags, float* Fx, float* Fy,
                            float* Fz, int nx, int ny, int nz, float gamma_lu, int wetting,
                            float theta);
void wo_compute_marangoni_force(const float* T, const float* phi, const float* f_l, float* Fx,
                                float* Fy, float* Fz, const int32_t* flags, int nx, int ny, int nz,
                                float dgamma);
void wo_apply_gas_shear_stress(float* Fx, float* Fy, const float* phi, const int32_t* flags,
                               int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                               float tau_peak_pa, float dt, float dx, float rho_ref);
void wo_apply_vapor_recoil(float* Fz, const float* T, const float* phi, const int32_t* flags,
                           int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                           float recoil_pa, float T_ref, float dt, float dx, float rho_ref);
void wo_apply_vapor_recoil_cc(float* Fz, const float* T, const float* phi, const int32_t* flags,
                              int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                              float P_ref, float T_boil, float L_vap, float R_spec, float C_acc,
                              float dt, float dx, float rho_ref);
void wo_apply_arc_pressure(float* Fz, const int32_t* flags, const float* phi, int nx, int ny,
                           int nz, float arc_i, float arc_j, float arc_k, float sigma,
                           float pressure, float dt, float dx, float rho_ref);
void wo_add_hydrostatic_gravity(float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                                float rho_ref, float g_lu);
void wo_add_buoyancy(const float* T, float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                     float g_lu, float beta, float T_ref, float rho_ref);
void wo_clamp_body_force_magnitude(float* Fx, float* Fy, float* Fz, const int32_t* flags,
                                   int64_t n, float F_max);
void wo_collide_mrt(const float* f_src, float* f_dst, float* rho, float* ux, float* uy, float* uz,
                    const float* Fx, const float* Fy, const float* Fz, const float* f_l,
                    const int32_t* flags, int64_t n, float omega_s, float omega_b,
                    float C_darcy);
void wo_collide_srt(const float* f_src, float* f_dst, float* rho, float* ux, float* uy, float* uz,
                    const float* Fx, const float* Fy, const float* Fz, const float* f_l,
                    const int32_t* flags, int64_t n, float omega, float C_darcy);
void wo_clamp_velocity_mach(float* ux, float* uy, float* uz, const int32_t* flags, int64_t n,
                            float u_max);
void wo_stream(const float* f_src, float* f_dst, const int32_t* flags, int nx, int ny, int nz);
void wo_update_time_above_T(const float* T, const int32_t* flags, float* t800, float* t1100,
                            float* tsol, int64_t n, float dt, float T800, float T1100, float Tsol);
void wo_snapshot_forces(const float* Fx, const float* Fy, const float* Fz, float* Sx, float* Sy,
                        float* Sz, int64_t n);
void wo_remelt_hot_solid_scalar(const float* T, float* H, float* f_l, float* phi, int32_t* flags,
                                int64_t n, float cp_rho, float Ts, float Tl, float L_rho);
void wo_solidify_trailing_pool_scalar(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                                      float* ux, float* uy, float* uz, int nx, int ny, int nz,
                                      float cp_rho, float arc_i, float arc_j, float arc_k,
                                      float dir_x, float dir_y, float dir_z, float lookback,
                                      float T_freeze, float Ts);
void wo_solidify_cooled_metal(const float* T, float* f_l, float* phi, int32_t* flags, float* ux,
                              float* uy, float* uz, int64_t n, float Ts, int zero_velocity);
float wo_surface_height_at(const float* phi, const int32_t* flags, int nx, int ny, int nz, int i0,
                           int j0, int nz_fallback);
void wo_feed_wire(float* f_src, int32_t* flags, float* f_l, float* phi, float* H, float* T,
                  float* rho, int nx, int ny, int nz, float arc_i, float arc_j, float arc_k,
                  float drop_r, float target_vol, float T_drop, float cp_rho, float L_rho,
                  float rho0, float* vol_acc, float cell_vol);
void wo_feed_wire_momentum(float* uz, const int32_t* flags, const float* f_l, int nx, int ny,
                           int nz, float arc_i, float arc_j, float arc_k, float drop_r,
                           float vz_lu);
void wo_feed_wire_surface(float* f_src, int32_t* flags, float* f_l, float* phi, float* H,
                          float* T, float* rho, int nx, int ny, int nz, float arc_i, float arc_j,
                          float arc_k, float foot_r, float drop_r, float target_vol, float T_drop,
                          float cp_rho, float L_rho, float rho0, float* vol_acc, float* real_acc,
                          float cell_vol);
void wo_feed_wire_momentum_impact(float* f_src, const float* rho, float* ux, float* uy, float* uz,
                                  const int32_t* flags, const float* f_l, int nx, int ny, int nz,
                                  float arc_i, float arc_j, float arc_k, float drop_r, float vx,
                                  float vy, float vz);
void wo_apply_droplet_impact_pressure(float* Fz, const int32_t* flags, const float* phi,
                                      const float* f_l, int nx, int ny, int nz, float arc_i,
                                      float arc_j, float arc_k, float drop_r, float impact_pa,
                                      float dt, float dx, float rho_ref);
/* Lorentz (config-5) kernels */
void wo_elec_build_sigma(float* sigma, const float* f_l, const int32_t* flags, int64_t n,
                         float s_liq, float s_sol);
void wo_elec_inject_arc_source(float* src, int nx, int ny, int nz, float arc_i, float arc_j,
                               float arc_k, float sigma_cells, float current, float dx);
void wo_elec_normalize_source(float* src, int64_t n, float current, float dx);
void wo_elec_jacobi_step(const float* phi_in, float* phi_out, const float* sigma,
                         const float* src, const int32_t* flags, int nx, int ny, int nz, float dx,
                         float omega_j, int nz_solid);
void wo_elec_l1_diff(const float* a, const float* b, int64_t n, double* diff, double* norm);
void wo_elec_compute_J(float* Jx, float* Jy, float* Jz, const float* phi, const float* sigma,
                       const int32_t* flags, int nx, int ny, int nz, float dx);
void wo_elec_bins(const float* Jz, float* bins, int nx, int ny, int nz, float arc_i, float arc_j,
                  float dx, float bin_dr, int n_bins);
void wo_elec_B_axisymmetric(float* Bx, float* By, float* Bz, const float* bins, int nx, int ny,
                            int nz, float arc_i, float arc_j, float dx, float bin_dr, float mu0,
                            int n_bins);
void wo_apply_lorentz_JxB(float* Fx, float* Fy, float* Fz, const float* Jx, const float* Jy,
                          const float* Jz, const float* Bx, const float* By, const float* Bz,
                          const float* f_l, const int32_t* flags, int64_t n, float dt, float dx,
                          float rho_ref);

/* material-table path (kernels.py:1686-2010, 2221-2269, 2454-2570, 2889-2965) */
void wo_refresh_thermal_properties(const float* T, float* cp_f, float* alpha_f, float* dg_f,
                                   float* tau_f, const int32_t* flags, int64_t n,
                                   const float* tab, const int32_t* cnt, const float* fb,
                                   const float* ref, float rho, float dt, float dx,
                                   float force_scale, float marangoni_scale);
void wo_advect_diffuse_temperature_variable(float* H, const float* T, const float* ux,
                                            const float* uy, const float* uz,
                                            const int32_t* flags, const float* alpha_f,
                                            const float* cp_f, int nx, int ny, int nz, float dt);
void wo_update_phase_variable_cp(const float* H, float* T, float* f_l, const float* cp_f,
                                 int64_t n, float L_rho, float Ts, float Tl, float H_sol,
                                 float H_liq);
void wo_clamp_enthalpy_ceiling_variable_cp(float* H, const int32_t* flags, const float* cp_f,
                                           int64_t n, float H_liq, float Tl, float T_cap);
void wo_clamp_enthalpy_floor(float* H, const float* cp_f, const int32_t* flags, int64_t n,
                             float T_floor);
void wo_compute_marangoni_force_variable(const float* T, const float* phi, const float* f_l,
                                         float* Fx, float* Fy, float* Fz, const int32_t* flags,
                                         const float* dg_f, int nx, int ny, int nz);
void wo_collide_srt_variable_tau(const float* f_src, float* f_dst, float* rho, float* ux,
                                 float* uy, float* uz, const float* Fx, const float* Fy,
                                 const float* Fz, const float* f_l, const int32_t* flags,
                                 const float* tau_f, int64_t n, float C_darcy);
void wo_remelt_hot_solid(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                         const float* cp_f, int64_t n, float Ts, float Tl, float L_rho);
void wo_solidify_trailing_pool(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                               float* ux, float* uy, float* uz, const float* cp_f, int nx, int ny,
                               int nz, float arc_i, float arc_j, float arc_k, float dir_x,
                               float dir_y, float dir_z, float lookback, float T_freeze,
                               float Ts);

/* kernels.py:3182-3205 inject_tracers with the library's counter-based hash
 * (the reference's ti.random() is not reproducible) */
void wo_inject_tracers(float* pos, int32_t* active, int32_t* head, int max_tracers, float arc_x,
                       float arc_y, float arc_z, float sigma_m, int spawn_count, uint64_t seed);
/* kernels.py:3207-3255 advect_tracers */
void wo_advect_tracers(float* pos, int32_t* active, const float* ux, const float* uy,
                       const float* uz, const float* f_l, const int32_t* flags, int nx, int ny,
                       int nz, float dx, int max_tracers);

/* kernels.py:2620-2723 shift_simulation_window_x */
void wo_shift_simulation_window_x(float* f_a, float* f_b, float* T, float* H, float* f_l,
                                  float* phi, int32_t* flags, float* T_max, float* T_prev,
                                  float* dT_dt, float* t800, float* t1100, float* tsol,
                                  float* rho, float* ux, float* uy, float* uz, float* Fx,
                                  float* Fy, float* Fz, float* cp_f, float* alpha_f,
                                  float* dg_f, float* tau_f, int n_shift, float T_amb,
                                  float cp_rho, float rho0, int nz_solid, int nx, int ny, int nz);

/* kernels.py:3354-3376 compute_curvature_field */
void wo_compute_curvature_field(const float* phi, const int32_t* flags, float* kappa, int nx,
                                int ny, int nz);
/* kernels.py:3379-3418 compute_vorticity_magnitude */
void wo_compute_vorticity_magnitude(const float* ux, const float* uy, const float* uz,
                                    const int32_t* flags, float* vort, int nx, int ny, int nz,
                                    float dt);

#ifdef __cplusplus
}
#endif
#endif
