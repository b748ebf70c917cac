/* waam_b200 -- C ABI of the B200 (sm_100a) coupled melt-pool step.
 *
 * Drop-in native backend for the waam_twin operator API (the physics modules) and
 * its step driver (solvers/coupled_step.py:73-464) of THEDARKDEACON/waam_solver.
 * All pointers are DEVICE pointers to memory owned by the caller (torch
 * tensors in the Python host); the library never allocates or frees on these
 * paths.  `stream` is a cudaStream_t passed as void*; every call is
 * asynchronous and stream-ordered.  Sizes: scalar fields hold nx*ny*nz
 * elements (k fastest), population fields 19*nx*ny*nz, flags are int32 with
 * FLUID=0, SOLID=1, GAS=2, IFACE=4 (grid.py:63-66).
 *
 * Every call returns WAAM_OK (0) or a negative status; waam_last_error()
 * gives the message of the last failure on the calling thread.  Entry points
 * that reduce over the grid need a workspace of waam_workspace_bytes(n)
 * bytes (device memory, 256-byte aligned), which the caller allocates once.
 */
#ifndef WAAM_B200_H
#define WAAM_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define WAAM_OK 0
#define WAAM_ERR_INVALID -1   /* bad argument (null pointer, size, workspace) */
#define WAAM_ERR_CUDA -2      /* CUDA launch / runtime error */
#define WAAM_ERR_DEVICE -3    /* a kernel reported a failed device-side check */

const char* waam_last_error(void);
int waam_abi_version(void);
/* Bytes of device workspace needed by the reducing entry points and the fused
 * step for a grid of n cells (block partial sums and a field-sized scratch). */
size_t waam_workspace_bytes(int64_t n);
/* sizeof of the ABI structs, for FFI layout checks: 0 WaamFields,
 * 1 WaamStepParams, 2 WaamMaterialTables, 3 WaamTelemetry, 4 WaamProbeSet,
 * 5 WaamShiftPlane, 6 WaamExportChannel (0 for any other value) */
size_t waam_struct_size(int which);

/* ---- operator API: one entry per reference Taichi kernel ---------------- */

/* kernels.py:62-120 init_grid (called by WAAMTwin.reset, twin.py:486-531) */
int waam_init_grid(float* f, float* rho, float* ux, float* uy, float* uz, float* T, float* H,
                   float* f_l, float* phi, int32_t* flags, int nx, int ny, int nz, float T_amb,
                   float rho0, float cp_rho, int nz_solid, int pi0, int pi1, int pj0, int pj1,
                   void* stream);
/* kernels.py:161-170 clear_forces (physics/forces.py:104) */
int waam_clear_forces(float* Fx, float* Fy, float* Fz, int64_t n, void* stream);
/* kernels.py:443-510 inject_arc_heat (physics/arc.py:63-72 Gaussian2D, 128-137 conical).
 * Writes the weight sum to norm_buf (device float, grid.py:163 arc_norm_buf). */
int waam_inject_arc_heat(float* H, const int32_t* flags, const float* f_l, float* norm_buf,
                         int nx, int ny, int nz, float arc_i, float arc_j, float arc_k, float Q_w,
                         float sigma, float dt, float dx3, float eta, float pen, int enable,
                         void* workspace, size_t workspace_bytes, void* stream);
/* kernels.py:548-622 inject_goldak_heat (physics/arc.py:106-119 Goldak3D) */
int waam_inject_goldak_heat(float* H, const int32_t* flags, const float* f_l, float* norm_buf,
                            int nx, int ny, int nz, float arc_i, float arc_j, float arc_k,
                            float Q_w, float dt, float dx3, float eta, float sign, float ff,
                            float fr, float a_f, float a_r, float b, float c, float pen,
                            int enable, void* workspace, size_t workspace_bytes, void* stream);
/* The operation of waam_inject_goldak_heat, for callers that cannot allocate
 * device memory (an FFI host without a CUDA allocator, or a step loop under a
 * fixed device-memory budget): its reduction scratch is a static device array
 * inside the library, so it takes no workspace.  The result equals
 * waam_inject_goldak_heat's to rounding: its double weight sum is split over
 * ceil(n / 2048) blocks instead of the workspace path's fixed block count, so
 * the float32 weight sum can differ in the last bit.  No counterpart in the
 * reference.  Grids above 16,777,216 cells are rejected
 * with WAAM_ERR_INVALID; calls that overlap on the GPU race on the shared
 * scratch; the first call on a device resolves the scratch address and
 * should come before any stream capture. */
int waam_inject_goldak_heat_noalloc(float* H, const int32_t* flags, const float* f_l,
                                    float* norm_buf, int nx, int ny, int nz, float arc_i,
                                    float arc_j, float arc_k, float Q_w, float dt, float dx3,
                                    float eta, float sign, float ff, float fr, float a_f,
                                    float a_r, float b, float c, float pen, int enable,
                                    void* stream);
/* kernels.py:1953-1984 clamp_enthalpy_ceiling_scalar (physics/thermal.py:30) */
int waam_clamp_enthalpy_ceiling_scalar(float* H, const int32_t* flags, int64_t n, float cp_rho,
                                       float Ts, float Tl, float T_cap, float L_rho, void* stream);
/* kernels.py:1611-1682 advect_diffuse_temperature (physics/thermal.py:16); neighbour
 * reads see H from before the call (snapshot kept in the workspace). */
int waam_advect_diffuse_temperature(float* H, const float* T, const float* ux, const float* uy,
                                    const float* uz, const int32_t* flags, int nx, int ny, int nz,
                                    float alpha_lu, float dt, float cp_rho, void* workspace,
                                    size_t workspace_bytes, void* stream);
/* kernels.py:1519-1556 update_phase (physics/phase_change.py:5) */
int waam_update_phase(const float* H, float* T, float* f_l, int64_t n, float cp_rho,
                      float L_rho, float Ts, float Tl, void* stream);
/* kernels.py:3016-3032 update_T_max (physics/thermal.py:21) */
int waam_update_T_max(const float* T, float* T_max, const int32_t* flags, int64_t n,
                      void* stream);
/* kernels.py:2013-2027 update_cooling_rate (physics/thermal.py:22) */
int waam_update_cooling_rate(const float* T, float* T_prev, float* dT_dt, const int32_t* flags,
                             int64_t n, float dt_phys, void* stream);
/* kernels.py:2030-2082 apply_thermal_boundary_losses (physics/thermal.py:18) */
int waam_apply_thermal_boundary_losses(float* H, const float* T, const int32_t* flags, int nx,
                                       int ny, int nz, float T_amb, float h_conv, float eps_rad,
                                       int conv, int rad, float dt, float dx, float sigma_sb,
                                       void* stream);
/* kernels.py:1937-1950 clamp_enthalpy_floor_scalar (physics/thermal.py:29) */
int waam_clamp_enthalpy_floor_scalar(float* H, float cp_rho, const int32_t* flags, int64_t n,
                                     float T_floor, void* stream);
/* kernels.py:2320-2361 advect_phi (physics/free_surface.py:62) */
int waam_advect_phi(float* phi_dst, const float* phi_src, const float* ux, const float* uy,
                    const float* uz, const int32_t* flags, int nx, int ny, int nz, void* stream);
/* kernels.py:2364-2391 reinitialize_phi (physics/free_surface.py:63) */
int waam_reinitialize_phi(float* phi, const int32_t* flags, int64_t n, void* stream);
/* kernels.py:933-991 apply_contact_angle_phi_bc (physics/free_surface.py:67); sequential
 * in k inside a column, other columns read from the pre-call snapshot. */
int waam_apply_contact_angle_phi_bc(float* phi, const int32_t* flags, int nx, int ny, int nz,
                                    float theta, void* workspace, size_t workspace_bytes,
                                    void* stream);
/* kernels.py:2394-2419 update_flags_from_phi (physics/free_surface.py:64) */
int waam_update_flags_from_phi(const float* phi, const float* f_l, int32_t* flags, int nx,
                               int ny, int nz, int nz_solid, void* stream);
/* kernels.py:3484-3504 sync_phi_liquid_fraction (physics/free_surface.py:65) */
int waam_sync_phi_liquid_fraction(const float* phi, float* f_l, const int32_t* flags, int64_t n,
                                  void* stream);
/* kernels.py:858-926 compute_csf_tension (physics/forces.py:114-133) */
int waam_compute_csf_tension(const float* phi, const int32_t* flags, float* Fx, float* Fy,
                             float* Fz, int nx, int ny, int nz, float gamma_lu, int wetting,
                             float theta, void* stream);
/* kernels.py:2158-2217 compute_marangoni_force (physics/forces.py:105) */
int waam_compute_marangoni_force(const float* T, const float* phi, const float* f_l, float* Fx,
                                 float* Fy, float* Fz, const int32_t* flags, int nx, int ny,
                                 int nz, float dgamma, void* stream);
/* kernels.py:3038-3083 apply_arc_pressure (physics/forces.py:110) */
/* kernels.py:1094-1141 apply_gas_shear_stress (its arc_k argument is unused) */
int waam_apply_gas_shear_stress(float* Fx, float* Fy, const float* phi, const int32_t* flags,
                                int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                                float tau_peak_pa, float dt, float dx, float rho_ref,
                                void* stream);
/* kernels.py:995-1028 apply_vapor_recoil (T-ratio form) */
int waam_apply_vapor_recoil(float* Fz, const float* T, const float* phi, const int32_t* flags,
                            int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                            float recoil_pa, float T_ref, float dt, float dx, float rho_ref,
                            void* stream);
/* kernels.py:1046-1091 apply_vapor_recoil_clausius_clapeyron */
int waam_apply_vapor_recoil_cc(float* Fz, const float* T, const float* phi, const int32_t* flags,
                               int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                               float P_ref, float T_boil, float L_vap, float R_spec, float C_acc,
                               float dt, float dx, float rho_ref, void* stream);
int waam_apply_arc_pressure(float* Fz, const int32_t* flags, const float* phi, int nx, int ny,
                            int nz, float arc_i, float arc_j, float arc_k, float sigma,
                            float pressure, float dt, float dx, float rho_ref, void* stream);
/* kernels.py:2756-2772 add_hydrostatic_gravity (physics/forces.py:109) */
int waam_add_hydrostatic_gravity(float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                                 float rho_ref, float g_lu, void* stream);
/* kernels.py:2729-2753 add_buoyancy (physics/forces.py:108) */
int waam_add_buoyancy(const float* T, float* Fz, const float* f_l, const int32_t* flags,
                      int64_t n, float g_lu, float beta, float T_ref, float rho_ref,
                      void* stream);
/* kernels.py:3286-3309 clamp_body_force_magnitude (solvers/coupled_step.py:356-362) */
int waam_clamp_body_force_magnitude(float* Fx, float* Fy, float* Fz, const int32_t* flags,
                                    int64_t n, float F_max, void* stream);
/* cumulant_kernel.py:28-209 collide_mrt (physics/lbm.py:9) */
int waam_collide_mrt(const float* f_src, float* f_dst, float* rho, float* ux, float* uy,
                     float* uz, const float* Fx, const float* Fy, const float* Fz,
                     const float* f_l, const int32_t* flags, int64_t n, float omega_s,
                     float omega_b, float C_darcy, void* stream);
/* kernels.py:2778-2885 collide_srt (physics/lbm.py:6) */
int waam_collide_srt(const float* f_src, float* f_dst, float* rho, float* ux, float* uy,
                     float* uz, const float* Fx, const float* Fy, const float* Fz,
                     const float* f_l, const int32_t* flags, int64_t n, float omega,
                     float C_darcy, void* stream);
/* kernels.py:3312-3335 clamp_velocity_mach (solvers/coupled_step.py:398-402) */
int waam_clamp_velocity_mach(float* ux, float* uy, float* uz, const int32_t* flags, int64_t n,
                             float u_max, void* stream);
/* kernels.py:2971-3010 stream (physics/lbm.py:8) */
int waam_stream(const float* f_src, float* f_dst, const int32_t* flags, int nx, int ny, int nz,
                void* stream);
/* kernels.py:3261-3283 update_time_above_T (solvers/coupled_step.py:418-423) */
int waam_update_time_above_T(const float* T, const int32_t* flags, float* t800, float* t1100,
                             float* tsol, int64_t n, float dt, float T800, float T1100,
                             float Tsol, void* stream);
/* kernels.py:3338-3350 snapshot_forces (solvers/coupled_step.py:424) */
int waam_snapshot_forces(const float* Fx, const float* Fy, const float* Fz, float* Sx, float* Sy,
                         float* Sz, int64_t n, void* stream);
/* kernels.py:2489-2520 remelt_hot_solid_scalar (physics/free_surface.py:69) */
int waam_remelt_hot_solid_scalar(const float* T, float* H, float* f_l, float* phi,
                                 int32_t* flags, int64_t n, float cp_rho, float Ts, float Tl,
                                 float L_rho, void* stream);
/* kernels.py:2573-2617 solidify_trailing_pool_scalar (solvers/coupled_step.py:452-457) */
int waam_solidify_trailing_pool_scalar(float* T, float* H, float* f_l, float* phi,
                                       int32_t* flags, float* ux, float* uy, float* uz, int nx,
                                       int ny, int nz, float cp_rho, float arc_i, float arc_j,
                                       float arc_k, float dir_x, float dir_y, float dir_z,
                                       float lookback, float T_freeze, float Ts, void* stream);
/* kernels.py:2422-2450 solidify_cooled_metal (physics/free_surface.py:73-91) */
int waam_solidify_cooled_metal(const float* T, float* f_l, float* phi, int32_t* flags,
                               float* ux, float* uy, float* uz, int64_t n, float Ts,
                               int zero_velocity, void* stream);
/* kernels.py:625-641 surface_height_at (physics/free_surface.py:66); writes the
 * height to out (device float, grid.py:160 surface_k_buf). */
int waam_surface_height_at(const float* phi, const int32_t* flags, float* out, int nx, int ny,
                           int nz, int i0, int j0, int nz_fallback, void* stream);
/* kernels.py:278-400 feed_wire_surface (physics/deposition.py:247); serial
 * lexicographic budget order; vol_acc / real_acc are device floats
 * (grid.py:161-162 deposit_vol_buf / deposit_real_buf).  One CTA per call. */
int waam_feed_wire_surface(float* f_src, int32_t* flags, float* f_l, float* phi, float* H,
                           float* T, float* rho, int nx, int ny, int nz, float arc_i, float arc_j,
                           float arc_k, float foot_r, float drop_r, float target_vol,
                           float T_drop, float cp_rho, float L_rho, float rho0, float* vol_acc,
                           float* real_acc, float cell_vol, void* stream);
/* kernels.py:177-242 feed_wire (physics/deposition.py:22): the older droplet
 * feed -- GAS cells inside the droplet sphere or the column above the arc
 * become liquid metal while the volume budget *vol_acc (device float) is below
 * target_vol, in serial lexicographic order.  f_src holds populations in the
 * storage f_storage (as WaamStepParams.f_storage).  One CTA per call. */
int waam_feed_wire(void* f_src, int f_storage, int32_t* flags, float* f_l, float* phi, float* H,
                   float* T, float* rho, int nx, int ny, int nz, float arc_i, float arc_j,
                   float arc_k, float drop_r, float target_vol, float T_drop, float cp_rho,
                   float L_rho, float rho0, float* vol_acc, float cell_vol, void* stream);
/* kernels.py:644-676 feed_wire_momentum (physics/deposition.py:24):
 * uz = min(uz + vz_lu, 0.15) for the non-gas cells with f_l >= 0.5 of the
 * droplet's column. */
int waam_feed_wire_momentum(float* uz, const int32_t* flags, const float* f_l, int nx, int ny,
                            int nz, float arc_i, float arc_j, float arc_k, float drop_r,
                            float vz_lu, void* stream);
/* The droplet's whole deposition, solvers/coupled_step.py:126-151: attempt t
 * is feed_wire_surface with footprint radius foot_radii[t]; attempt 0 starts
 * from *vol_acc / *real_acc, attempt t > 0 runs only while the converted
 * volume *real_acc is below accept_volume (compared in double) and starts
 * with both budgets at that volume.  One launch, no host round trip between
 * attempts; read *real_acc afterwards for the placed volume.  f_src holds
 * populations in the storage f_storage (as WaamStepParams.f_storage). */
#define WAAM_DEPOSIT_MAX_TRIES 16
int waam_deposit_droplet(void* f_src, int f_storage, int32_t* flags, float* f_l, float* phi,
                         float* H, float* T, float* rho, int nx, int ny, int nz, float arc_i,
                         float arc_j, float arc_k, const float* foot_radii, int n_tries,
                         double accept_volume, float drop_r, float target_vol, float T_drop,
                         float cp_rho, float L_rho, float rho0, float* vol_acc, float* real_acc,
                         float cell_vol, void* stream);
/* kernels.py:1176-1233 feed_wire_momentum_impact (physics/weld_forces.py:534-542) */
int waam_feed_wire_momentum_impact(float* f_src, const float* rho, float* ux, float* uy,
                                   float* uz, const int32_t* flags, const float* f_l, int nx,
                                   int ny, int nz, float arc_i, float arc_j, float arc_k,
                                   float drop_r, float vx, float vy, float vz, void* stream);
/* feed_wire_momentum_impact on populations in any storage (f_storage as
 * WaamStepParams.f_storage); no counterpart in the reference, which stores
 * float32 only. */
int waam_feed_wire_momentum_impact_stored(void* f_src, int f_storage, const float* rho, float* ux,
                                          float* uy, float* uz, const int32_t* flags,
                                          const float* f_l, int nx, int ny, int nz, float arc_i,
                                          float arc_j, float arc_k, float drop_r, float vx,
                                          float vy, float vz, void* stream);
/* kernels.py:1142-1173 apply_droplet_impact_pressure (physics/weld_forces.py:543-550) */
int waam_apply_droplet_impact_pressure(float* Fz, const int32_t* flags, const float* phi,
                                       const float* f_l, int nx, int ny, int nz, float arc_i,
                                       float arc_j, float arc_k, float drop_r, float impact_pa,
                                       float dt, float dx, float rho_ref, void* stream);

/* ---- Lorentz force of the welding current (physics/weld_forces.py:196-281) -- */

/* kernels.py:1237-1251 elec_build_sigma */
int waam_elec_build_sigma(float* sigma, const float* f_l, const int32_t* flags, int64_t n,
                          float sigma_liquid, float sigma_solid, void* stream);
/* kernels.py:1255-1284 elec_clear_source + elec_inject_arc_source (one pass) */
int waam_elec_inject_arc_source(float* source, int nx, int ny, int nz, float arc_i, float arc_j,
                                float arc_k, float sigma_cells, float current_A, float dx,
                                void* stream);
/* elec_clear_source + elec_inject_arc_source + elec_normalize_source
 * (kernels.py:1255-1301, as physics/weld_forces.py:206-211 calls them) in two
 * passes that read nothing: the normalising sum over the source's k slab,
 * then every cell written once with its scaled value. */
int waam_elec_arc_source(float* source, int nx, int ny, int nz, float arc_i, float arc_j,
                         float arc_k, float sigma_cells, float current_A, float dx,
                         void* workspace, size_t workspace_bytes, void* stream);
/* waam_elec_arc_source with the arc height read from device memory */
int waam_elec_arc_source_dev(float* source, int nx, int ny, int nz, float arc_i, float arc_j,
                             const float* arc_k_dev, float sigma_cells, float current_A,
                             float dx, void* workspace, size_t workspace_bytes, void* stream);
/* kernels.py:1288-1301 elec_normalize_source; the sum is taken in double */
int waam_elec_normalize_source(float* source, int64_t n, float target_current_A, float dx,
                               void* workspace, size_t workspace_bytes, void* stream);
/* elec_build_sigma plus a byte mask (fixed[c] = 1) of the cells the Jacobi
 * sweep holds at 0: GAS, and SOLID at k <= nz_solid (kernels.py:1315-1355) */
int waam_elec_build_sigma_mask(float* sigma, uint8_t* fixed, const float* f_l,
                               const int32_t* flags, int nx, int ny, int nz, float sigma_liquid,
                               float sigma_solid, int nz_solid, void* stream);
/* n_sweeps elec_jacobi_step sweeps ping-ponging phi_a -> phi_b -> phi_a ...,
 * the last one with elec_l1_diff of its output against its input into
 * diff_buf / norm_buf (physics/weld_forces.py:235-245, one check chunk): the
 * last iterate ends in phi_b for an odd n_sweeps, in phi_a for an even one.
 * fixed is the mask of waam_elec_build_sigma_mask; the source must be 0
 * outside the k slab of waam_elec_arc_source for (arc_k, sigma_cells). */
int waam_elec_jacobi_chunk(float* phi_a, float* phi_b, const float* sigma, const float* source,
                           const uint8_t* fixed, int nx, int ny, int nz, float dx, float omega_j,
                           int n_sweeps, float arc_k, float sigma_cells, float* diff_buf,
                           float* norm_buf, void* workspace, size_t workspace_bytes,
                           void* stream);
/* The potential solve over its live cells (those the sweep does not hold at
 * 0: neither GAS nor SOLID at k <= nz_solid).  waam_elec_prepare writes sigma
 * (elec_build_sigma) and the fixed-cell mask, zeroes phi_b at cells that
 * became fixed since the mask was last built (an all-zero mask: every fixed
 * cell), lists those cells (zero_list) and the live cells (live_list, in a
 * fixed order; counts[0] = live, counts[1] = newly fixed; counts has
 * waam_elec_counts_len entries).  waam_elec_jacobi_live runs n_sweeps sweeps
 * phi_a -> phi_b -> ... over the live list, the last with the L1 check; with
 * first_chunk set (the first call of a solve, phi_a its input) it also zeroes
 * the newly fixed cells of phi_a after the first sweep.  Exact against the
 * full-grid sweeps as long as both buffers are only written by these calls
 * (and elec_init_ground) between mask builds: the fixed cells of both then
 * hold 0, which is what every sweep writes there.  The source's k slab
 * comes from the arc height at arc_k_dev (device memory, e.g. the fused
 * step's scalar 0), so the solve needs no host copy of it. */
int64_t waam_elec_counts_len(int nx, int ny, int nz);
int waam_elec_prepare(float* sigma, uint8_t* fixed, float* phi_b, const float* f_l,
                      const int32_t* flags, int nx, int ny, int nz, float sigma_liquid,
                      float sigma_solid, int nz_solid, int32_t* live_list, int32_t* zero_list,
                      int32_t* counts, int64_t counts_len, void* stream);
int waam_elec_jacobi_live(float* phi_a, float* phi_b, const float* sigma, const float* source,
                          const int32_t* live_list, const int32_t* zero_list,
                          const int32_t* counts, int nx, int ny, int nz, float dx,
                          float omega_j, int n_sweeps, int first_chunk, const float* arc_k_dev,
                          float sigma_cells, float* diff_buf, float* norm_buf, void* workspace,
                          size_t workspace_bytes, void* stream);
/* kernels.py:1304-1312 elec_init_ground (phi = 0) */
int waam_elec_init_ground(float* phi, int64_t n, void* stream);
/* kernels.py:1315-1355 elec_jacobi_step; phi_in and phi_out must differ */
int waam_elec_jacobi_step(const float* phi_in, float* phi_out, const float* sigma,
                          const float* source, const int32_t* flags, int nx, int ny, int nz,
                          float dx, float omega_j, int nz_solid, void* stream);
/* elec_jacobi_step followed by elec_l1_diff(phi_out, phi_in) (kernels.py:1387-1398)
 * in the same pass: *diff_buf = sum|phi_out - phi_in|, *norm_buf = sum|phi_in|. */
int waam_elec_jacobi_step_l1(const float* phi_in, float* phi_out, const float* sigma,
                             const float* source, const int32_t* flags, int nx, int ny, int nz,
                             float dx, float omega_j, int nz_solid, float* diff_buf,
                             float* norm_buf, void* workspace, size_t workspace_bytes,
                             void* stream);
/* kernels.py:1387-1398 elec_l1_diff: *diff_buf = sum|a - b|, *norm_buf = sum|b| */
int waam_elec_l1_diff(const float* a, const float* b, float* diff_buf, float* norm_buf, int nx,
                      int ny, int nz, void* workspace, size_t workspace_bytes, void* stream);
/* kernels.py:1358-1383 elec_compute_J */
int waam_elec_compute_J(float* Jx, float* Jy, float* Jz, const float* phi, const float* sigma,
                        const int32_t* flags, int nx, int ny, int nz, float dx, void* stream);
/* kernels.py:1402-1421 elec_bin_axial_current: bins (nz, n_bins) of Jz dx^2 by
 * radius; sums in double, stored as float */
int waam_elec_bin_axial_current(const float* Jz, float* bins, int nx, int ny, int nz, float arc_i,
                                float arc_j, float dx, float bin_dr_cells, int n_bins,
                                void* workspace, size_t workspace_bytes, void* stream);
/* kernels.py:1424-1435 elec_prefix_bins (float prefix over radius, in place) */
int waam_elec_prefix_bins(float* bins, int n_bins, int nz, void* stream);
/* kernels.py:1438-1475 elec_B_axisymmetric */
int waam_elec_B_axisymmetric(float* Bx, float* By, float* Bz, const float* bins, int nx, int ny,
                             int nz, float arc_i, float arc_j, float dx, float bin_dr_cells,
                             float mu0, int n_bins, void* stream);
/* After the potential solve (physics/weld_forces.py:261-276): elec_compute_J,
 * elec_bin_axial_current, elec_prefix_bins, elec_B_axisymmetric in one call */
int waam_elec_fields(float* Jx, float* Jy, float* Jz, float* Bx, float* By, float* Bz,
                     float* bins, const float* phi, const float* sigma, const int32_t* flags,
                     int nx, int ny, int nz, float arc_i, float arc_j, float dx,
                     float bin_dr_cells, float mu0, int n_bins, void* workspace,
                     size_t workspace_bytes, void* stream);
/* kernels.py:1479-1513 apply_lorentz_JxB */
int waam_apply_lorentz_JxB(float* Fx, float* Fy, float* Fz, const float* Jx, const float* Jy,
                           const float* Jz, const float* Bx, const float* By, const float* Bz,
                           const float* f_l, const int32_t* flags, int64_t n, float dt, float dx,
                           float rho_ref, void* stream);

/* ---- porosity tracers (kernels.py:3182-3255) ---------------------------- */

/* kernels.py:3182-3205 inject_tracers: spawn_count particles into consecutive
 * ring-buffer slots from *head (then *head += spawn_count), at random offsets
 * within +-sigma_m of (arc_x, arc_y), z = arc_z.  pos is (max_tracers, 3).
 * The offsets come from a counter-based hash of (seed, spawn index): the
 * reference's ti.random() stream is not reproducible, so a seed is added. */
int waam_inject_tracers(float* pos, int32_t* active, int32_t* head, int max_tracers, float arc_x,
                        float arc_y, float arc_z, float sigma_m, int spawn_count, uint64_t seed,
                        void* stream);
/* kernels.py:3207-3255 advect_tracers (nearest-cell velocity, pos += u*dx) */
int waam_advect_tracers(float* pos, int32_t* active, const float* ux, const float* uy,
                        const float* uz, const float* f_l, const int32_t* flags, int nx, int ny,
                        int nz, float dx, int max_tracers, void* stream);

/* ---- temperature-dependent material tables (kernels.py:1686-2010, 2454-2570) */

/* gpu_tables.py:12-80 MaterialGPUTables: up to 8 (T [K], value) knots per
 * property, sorted by T; a count of 0 selects the fallback constant.  The
 * struct is read on the host and passed to the kernels by value. */
#define WAAM_TABLE_KNOTS 8
typedef struct WaamMaterialTables {
    float cp_T[WAAM_TABLE_KNOTS], cp_V[WAAM_TABLE_KNOTS];
    float k_T[WAAM_TABLE_KNOTS], k_V[WAAM_TABLE_KNOTS];
    float mu_T[WAAM_TABLE_KNOTS], mu_V[WAAM_TABLE_KNOTS];
    float dgamma_T[WAAM_TABLE_KNOTS], dgamma_V[WAAM_TABLE_KNOTS];
    int32_t n_cp, n_k, n_mu, n_dgamma;
    float cp_fallback, k_fallback, mu_fallback, dgamma_fallback;
} WaamMaterialTables;

/* kernels.py:1710-1772 refresh_thermal_properties: per-cell rho*cp(T),
 * alpha_lu(T), dgamma_lu(T) (x force_scale x marangoni_scale) and SRT tau(T)
 * from the tables (use_tables = 1) or the reference constants; SOLID and GAS
 * cells take the reference constants.  `tables` is a host pointer. */
int waam_refresh_thermal_properties(const float* T, float* cp_rho_f, float* alpha_f,
                                    float* dgamma_f, float* tau_f, const int32_t* flags, int64_t n,
                                    const WaamMaterialTables* tables, float rho, float dt,
                                    float dx, float force_scale, float cp_rho_ref,
                                    float alpha_lu_ref, float dgamma_lu_ref, float tau_ref,
                                    float marangoni_scale, int use_tables, void* stream);
/* kernels.py:1775-1836 advect_diffuse_temperature_variable (snapshot of H in
 * the workspace, like waam_advect_diffuse_temperature) */
int waam_advect_diffuse_temperature_variable(float* H, const float* T, const float* ux,
                                             const float* uy, const float* uz,
                                             const int32_t* flags, const float* alpha_f,
                                             const float* cp_rho_f, int nx, int ny, int nz,
                                             float dt, void* workspace, size_t workspace_bytes,
                                             void* stream);
/* kernels.py:1839-1863 update_phase_variable_cp */
int waam_update_phase_variable_cp(const float* H, float* T, float* f_l, const float* cp_rho_f,
                                  int64_t n, float L_rho, float T_solidus, float T_liquidus,
                                  float H_sol, float H_liq, void* stream);
/* kernels.py:1988-2010 clamp_enthalpy_ceiling_variable_cp */
int waam_clamp_enthalpy_ceiling_variable_cp(float* H, const int32_t* flags, const float* cp_rho_f,
                                            int64_t n, float H_liq, float T_liquidus,
                                            float T_cap, void* stream);
/* kernels.py:1922-1935 clamp_enthalpy_floor (per-cell rho*cp) */
int waam_clamp_enthalpy_floor(float* H, const float* cp_rho_f, const int32_t* flags, int64_t n,
                              float T_floor, void* stream);
/* kernels.py:2221-2269 compute_marangoni_force_variable (per-cell dgamma) */
int waam_compute_marangoni_force_variable(const float* T, const float* phi, const float* f_l,
                                          float* Fx, float* Fy, float* Fz, const int32_t* flags,
                                          const float* dgamma_f, int nx, int ny, int nz,
                                          void* stream);
/* kernels.py:2889-2965 collide_srt_variable_tau: omega = 1 / (tau + 1e-6) per cell */
int waam_collide_srt_variable_tau(const float* f_src, float* f_dst, float* rho, float* ux,
                                  float* uy, float* uz, const float* Fx, const float* Fy,
                                  const float* Fz, const float* f_l, const int32_t* flags,
                                  const float* tau_f, int64_t n, float C_darcy, void* stream);
/* kernels.py:2454-2485 remelt_hot_solid (per-cell rho*cp) */
int waam_remelt_hot_solid(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                          const float* cp_rho_f, int64_t n, float T_solidus, float T_liquidus,
                          float L_rho, void* stream);
/* kernels.py:2524-2570 solidify_trailing_pool (per-cell rho*cp) */
int waam_solidify_trailing_pool(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                                float* ux, float* uy, float* uz, const float* cp_rho_f, int nx,
                                int ny, int nz, float arc_i, float arc_j, float arc_k, float dir_x,
                                float dir_y, float dir_z, float lookback, float T_freeze,
                                float T_solidus, void* stream);

/* ---- telemetry (twin.py:706-821; kernels.py:3424-3481) -------------------- */

#define WAAM_TOE_CELLS 16
/* Pool aggregates written by waam_telemetry_pool into device memory. */
typedef struct WaamTelemetry {
    double T_global;        /* max T over all cells, at least 0 */
    double T_peak;          /* max T over cells with f_l > 0.5, at least 0 */
    double peak_cool;       /* max -dT/dt over cells with phi > 0.05, at least 0 */
    double u2_max;          /* max |u|^2 (lattice units) over cells with f_l > 0.5 */
    double H_sum;           /* sum of H over all cells, FP64, fixed order */
    int64_t n_liquid;       /* cells with f_l > 0.5 */
    int64_t i_sum;          /* sum of their i (exact) */
    int32_t i_min, i_max;   /* their i extent (-1 without liquid) */
    int32_t i_c;            /* centroid slice round(i_sum / n_liquid) (half to even), clamped; -1 without liquid */
    int32_t y_min, y_max, z_min; /* extent of f_l > 0.5 in slice i_c (-1 when empty) */
    int32_t bead_k_max;     /* max k of SOLID cells with k >= nz_solid, -1 if none */
    int32_t n_tracers_active, n_tracers_trapped; /* porosity tracers with active == 1 / == 2 */
    int32_t toe_k0, toe_n;  /* toe-angle column (nx/3, ny/2, k0 .. k0 + toe_n - 1) */
    float toe_phi[WAAM_TOE_CELLS];
    int32_t toe_flags[WAAM_TOE_CELLS];
} WaamTelemetry;

/* kernels.py:3424-3468 telemetry_pool_reduce, the centroid slice of
 * twin.py:723-744 (kernels.py:3471-3481), the tracer counts, the bead height
 * of physics/electrical_stickout.py:39-50 and the toe column of
 * physics/bead_geometry.py:13-40, into `out` (device memory): two launches,
 * deterministic (FP64 enthalpy sum in a fixed order, integer sums exact).
 * H may be null (H_sum = 0), flags may be null (no bead height, no toe
 * column), tracer_active may be null (max_tracers ignored). */
int waam_telemetry_pool(const float* T, const float* f_l, const float* phi, const float* dT_dt,
                        const float* ux, const float* uy, const float* uz, const float* H,
                        const int32_t* flags, const int32_t* tracer_active, int max_tracers,
                        int nx, int ny, int nz, int nz_solid, WaamTelemetry* out,
                        void* workspace, size_t workspace_bytes, void* stream);

#define WAAM_MAX_PROBES 64
/* Probe cells (export/probes.py:29-37 resolve on the host; -1 = outside the grid). */
typedef struct WaamProbeSet {
    int32_t n_probes;
    int64_t cell[WAAM_MAX_PROBES];   /* (i * ny + j) * nz + k */
} WaamProbeSet;
/* export/probes.py:90-107: row[2p] = T, row[2p+1] = f_l at probe p (NaN outside).
 * `probes` is a host pointer, `row` device memory (2 * n_probes floats). */
int waam_probe_sample(const float* T, const float* f_l, const WaamProbeSet* probes, float* row,
                      void* stream);
/* physics/electrical_stickout.py:39-50: max k of SOLID cells with k >= nz_solid
 * into *out (device int32; -1 when there are none). */
int waam_bead_height(const int32_t* flags, int nx, int ny, int nz, int nz_solid, int32_t* out,
                     void* stream);

/* ---- moving window (kernels.py:2620-2723, twin.py:599-631) ---------------- */

#define WAAM_MAX_SHIFT_PLANES 64
#define WAAM_SHIFT_KEEP 0    /* moved, the right strip keeps its old values */
#define WAAM_SHIFT_CONST 1   /* moved, the right strip becomes `below` */
#define WAAM_SHIFT_BY_K 2    /* moved, the right strip becomes `below` for k < nz_solid, else `above` */
/* One field plane of nx*ny*nz elements (4-byte float / int32 or 16-bit), its
 * strip reset mode and the reset values as raw element bits. */
typedef struct WaamShiftPlane {
    void* ptr;
    int32_t elem_bytes;
    int32_t mode;
    uint32_t below;
    uint32_t above;
} WaamShiftPlane;
/* kernels.py:2620-2723 shift_simulation_window_x over any set of planes in one
 * launch: plane[i] = plane[i + n_shift] for i < nx - n_shift (the reference's
 * ascending in-place order), then the strip i >= nx - n_shift is reset per
 * plane.  `planes` is a host array (n_planes <= WAAM_MAX_SHIFT_PLANES);
 * n_shift >= 0. */
int waam_shift_window_x(const WaamShiftPlane* planes, int n_planes, int n_shift, int nx, int ny,
                        int nz, int nz_solid, void* stream);
/* twin.py:624-626: pos[:, 0] -= shift_m for every tracer slot */
int waam_shift_tracers_x(float* pos, int max_tracers, float shift_m, void* stream);

/* ---- export (export/vtk_io.py; kernels.py:3354-3418) ---------------------- */

/* kernels.py:3354-3376 compute_curvature_field: kappa = -div(n) (Brackbill) on
 * non-gas interior cells with |grad phi| >= 1e-6, else 0 */
int waam_compute_curvature_field(const float* phi, const int32_t* flags, float* kappa_out, int nx,
                                 int ny, int nz, void* stream);
/* kernels.py:3379-3418 compute_vorticity_magnitude: |curl u| / dt [1/s] on
 * non-gas cells (dx is accepted and unused, as in the reference) */
int waam_compute_vorticity_magnitude(const float* ux, const float* uy, const float* uz,
                                     const int32_t* flags, float* vort_out, int nx, int ny, int nz,
                                     float dx, float dt, void* stream);

#define WAAM_MAX_EXPORT_CHANNELS 48
/* channel operations, float32 arithmetic in the written order */
#define WAAM_EXPORT_COPY 0       /* src0 */
#define WAAM_EXPORT_COPY_I32 1   /* src0 as int32 */
#define WAAM_EXPORT_ADD 2        /* src0 + a */
#define WAAM_EXPORT_NEG 3        /* -src0 */
#define WAAM_EXPORT_LU_VEL 4     /* src0 * a / b            (a = dx, b = dt) */
#define WAAM_EXPORT_LU_ACC 5     /* src0 * a / b / b */
#define WAAM_EXPORT_SPEED 6      /* |(src0, src1, src2) * a / b| */
#define WAAM_EXPORT_ACC_MAG 7    /* |(src0, src1, src2) * a / b / b| */
#define WAAM_EXPORT_PRESSURE 8   /* (src0 - 1) * a * b * c */
#define WAAM_EXPORT_MUSHY 9      /* 1 where 0.05 < src0 < 0.95, else 0 */
typedef struct WaamExportChannel {
    int32_t op;
    float a, b, c;
    const void* src[3];
} WaamExportChannel;
/* One launch: channel q of the output (out + q * n, 4-byte elements) holds the
 * channel's value at every cell in VTK cell order, index i + nx * (j + ny * k).
 * `channels` is a host array (n_channels <= WAAM_MAX_EXPORT_CHANNELS); `out`
 * is device memory of n_channels * nx * ny * nz * 4 bytes. */
/* export/vtk_io.py:180-224 (the phi = 0.5 surface).  waam_cell_to_point:
 * values at the (nx+1)(ny+1)(nz+1) cell corners, each the mean of the cells
 * sharing it, for up to four fields (c1..c3 may be null; point index
 * (I * (ny+1) + J) * (nz+1) + K).  waam_isosurface: marching tetrahedra of
 * iso_points at `iso` (six tetrahedra per cube around its 0-7 diagonal);
 * per triangle vertex the edge key keys[3t + v] (lower point index times
 * the point count plus the upper one) and vals[(3t + v) * 6 + ..] = x, y, z
 * (origin + spacing * lattice position) and a0..a2 interpolated (null: 0);
 * order[t] = cube * 16 + tetrahedron * 2 + part restores a fixed order;
 * *count receives the triangle total (rows past `capacity` are not written).
 * Triangles face from above iso to below. */
int waam_cell_to_point(const float* c0, const float* c1, const float* c2, const float* c3,
                       float* p0, float* p1, float* p2, float* p3, int nx, int ny, int nz,
                       void* stream);
int waam_isosurface(const float* iso_points, const float* a0, const float* a1, const float* a2,
                    int nx, int ny, int nz, float iso, float spacing, float ox, float oy,
                    float oz, int64_t* keys, float* vals, int64_t* order,
                    unsigned long long* count, int64_t capacity, void* stream);
int waam_export_pack(const WaamExportChannel* channels, int n_channels, int nx, int ny, int nz,
                     void* out, void* stream);

/* ---- fused step: the B200 pipeline of solvers/coupled_step.py:73-464 ----- */

typedef struct WaamFields {
    /* populations, elements per WaamStepParams.f_storage (float or 16-bit) */
    void* f_src;    /* read by this step's collide (grid.f_src) */
    void* f_dst;    /* written by collide, streamed back into f_src */
    float* rho;
    float* ux;
    float* uy;
    float* uz;
    float* T;       /* temperature at step start ... */
    float* T_next;  /* ... and after the step (buffers swap on the host) */
    float* H;
    float* H_next;
    float* f_l;
    float* phi;
    float* phi_tmp;
    int32_t* flags;
    float* T_max;
    float* T_prev;
    float* dT_dt;
    float* t800;
    float* t1100;
    float* tsol;
    float* Fx;      /* body force of the step (== the reference's F_snap) */
    float* Fy;
    float* Fz;
    float* step_scalars; /* device float[16]: [0] arc k, [1] weight sum, [2] energy/weight,
                            [4], [5] torch position (arc_i, arc_j) in cells -- written by
                            the caller before waam_step_pre (a 2-float H2D copy per step) */
    int nx, ny, nz;
    /* porosity tracers advected after the stream (kernels.py:3207-3255); a
     * null pos or max_tracers == 0 skips them */
    float* tracer_pos;        /* (max_tracers, 3) */
    int32_t* tracer_active;   /* (max_tracers) */
    int max_tracers;
    /* per-cell material properties (grid.py:146-149), read and written when
     * WaamStepParams.use_tables != 0, otherwise unused (may be null) */
    float* cp_rho_f;
    float* alpha_f;
    float* dgamma_f;
    float* tau_f;
    /* adjoint tape of the collision (null: off): for every active cell of
     * the step, its index (tape_cells[t]) and its 19 pre-collision populations
     * (tape_f[q * tape_cap + t], float32 storage only); *tape_count receives
     * the number of active cells.  A step with more than tape_cap active
     * cells writes none of them and sets *tape_count to -1. */
    float* tape_f;
    int32_t* tape_cells;
    int32_t* tape_count;
    int64_t tape_cap;
    /* current density J (A/m^2) and self field B (T) of the welding current
     * (physics/weld_forces.py:261-276), solved by the caller between
     * waam_step_main_stage 0 and 1; when set, the collision adds the J x B
     * force (kernels.py:1479-1513) after the other body forces and before
     * their clamp, as the reference's force assembly does
     * (solvers/coupled_step.py:352-362).  Null: no Lorentz force. */
    const float* lorentz_J[3];
    const float* lorentz_B[3];
    /* flag copies for the pipelined stream (null: none): waam_step_main's
     * column pass writes the step's flags also to flags_copy_w, and the
     * pending stream of the previous step (WaamStepParams.stream_prev) reads
     * flags_copy_r, the copy that step wrote -- so it may run on while the
     * column pass rewrites the flags, and is joined only before the
     * collision.  The caller alternates two buffers from step to step (three
     * with flags_copy_rr).  Quiet tiles' cells are written too (GAS). */
    int32_t* flags_copy_w;
    const int32_t* flags_copy_r;
    /* health word of the fused step (null: off), device uint32 that the
     * kernels OR bits into (WAAM_HEALTH_*): the thermal stage when a non-gas
     * cell's enthalpy is not finite, the collision when an active cell's
     * density or velocity is not finite or its density lies outside
     * [WaamStepParams.rho_lo, rho_hi].  Nothing clears it; the caller reads
     * it where it synchronises anyway and zeroes it when it wants. */
    uint32_t* status;
    /* quiet-tile skipping of the fused step (all null: every tile is worked).
     * Tiles are the 32 (k) x 8 (j) cell blocks of one x plane, numbered
     * t = (i * ceil(ny / 8) + j / 8) * ceil(nz / 32) + k / 32; a chunk is the
     * 32 cells of one (i, j) column inside a tile (column-chunk number
     * (i * ny + j) * ceil(nz / 32) + k / 32).  With WaamStepParams.tile_skip
     * set, waam_step_pre marks as quiet every tile whose cells and every cell
     * within two lattice steps of them are GAS, and that was all GAS at the
     * step before; the arc, thermal, VOF and column stages leave quiet tiles
     * alone (they are exact no-ops there).  The caller owns and zero-fills:
     *   tile_bits: ceil(nz/32) * nx * ny chunk bytes (bit 0: all GAS, 1: all
     *     GAS the pass before, 2 / 3: top / bottom two cells GAS, 4-5: passes
     *     in a row whose flag copies of the chunk were all GAS), then one work
     *     byte per tile;
     *   tile_list: 1 + tiles int32 (count, then the tiles to work; the
     *     column pass zeroes the count for the next step);
     *   tile_part: tiles doubles (per-tile arc weight sums).
     * They carry state from step to step: after changing the fields any
     * other way, run the next step with tile_skip = 0. */
    uint8_t* tile_bits;
    int32_t* tile_list;
    double* tile_part;
    /* the flag copy of the step before the one flags_copy_r holds, for the
     * lagged stream (WaamStepParams.hold_stream / stream_lag); with it the
     * caller rotates three buffers (w, r, rr) from step to step */
    const int32_t* flags_copy_rr;
    /* Compact copy of the collision's output (all null: off).  Under the
     * reference's buffer order (collide f_src -> f_dst at the active cells,
     * stream f_dst -> f_src, swap) a cell active in two consecutive steps
     * reads in the second exactly the populations its first collision wrote,
     * so each collision also writes them, in stored form, to a slot of
     * pop_cache_dst, and the next collision reads them from pop_cache_src
     * (WaamStepParams.cache_read) in three or six 16-byte loads instead of
     * 19 scattered ones.  Slot: ((i*ny + j) * ceil(nz/32) + k/32) * 2 + the
     * cell's rank among the active cells of its 32-cell column chunk in k
     * order (ranks 0 and 1; the others go without); 96 bytes (4-byte
     * storage: 19 populations, cell index, stamp, pad) or 48 bytes (2-byte
     * storage: 19 populations, 2 bytes pad, cell index, stamp); a slot counts
     * only if its cell index and stamp match.  The caller allocates two
     * buffers of nx*ny*ceil(nz/32)*2 slots, each filled with 0xff bytes, and
     * swaps them with f_src / f_dst; pop_cache_stamp is one zeroed device
     * word that the thermal stage counts up once per step. */
    void* pop_cache_src;
    void* pop_cache_dst;
    uint32_t* pop_cache_stamp;
} WaamFields;

#define WAAM_HEALTH_NONFINITE_H 1u   /* H of a non-gas cell is NaN or infinite */
#define WAAM_HEALTH_NONFINITE_LBM 2u /* density or velocity of an active cell not finite */
#define WAAM_HEALTH_RHO_RANGE 4u     /* density of an active cell outside [rho_lo, rho_hi] */

typedef struct WaamStepParams {
    /* torch position (solvers/coupled_step.py:92-94); the kernels read it from
     * step_scalars[4..5], these copies are informational */
    float arc_i, arc_j;
    int welding;
    int nz_solid;
    /* arc source (physics/arc.py): kind 0 Gaussian/conical, 1 Goldak */
    int arc_kind;
    float arc_k_offset;  /* conical source: -1.5 (physics/arc.py:132) */
    float Q_w, eta, dt, dx, dx3, sigma_heat, sign, ff, fr, a_f, a_r, gb, gc, pen;
    int surface_weighting;
    /* thermal / phase (twin.py:244-274) */
    float cp_rho, L_rho, Ts, Tl, T_cap, alpha_lu;
    int cap_enabled;
    int heat_loss;
    float T_amb, h_conv, eps_rad, sigma_sb;
    int conv, rad;
    /* VOF */
    int vof, wetting;
    float theta;
    /* forces.  The fused step keeps F == 0 outside FLUID/IFACE cells; set
     * forces_from_buffer when F holds this step's droplet impact load (then F is
     * the starting force of active cells and stays untouched elsewhere), and
     * clear_forces when the previous step left F != 0 outside active cells. */
    int csf, hydro, forces_from_buffer, clear_forces;
    float gamma_lu, dgamma_lu, p_sigma, pressure, rho_phys, g_lu, beta, T_ref, F_cap;
    /* collision */
    int collision;  /* 0 MRT, 1 SRT */
    float omega, omega_b, C_darcy, u_cap;
    /* diagnostics and tail */
    float T800, T1100;
    int substrate_growth, bead_freeze;
    float dir_x, dir_y, dir_z, lookback, T_freeze;
    /* population storage of f_src / f_dst: 0 float32 f_q; 1 float16 and
     * 2 bfloat16 offsets f_q - w_q (rho0 = 1), rounded to nearest; the
     * arithmetic is float32 in every case */
    int f_storage;
    /* temperature-dependent material tables (twin.py:269-273): the thermal
     * stage refreshes WaamFields' property fields from T and then uses the
     * cell's own rho*cp and alpha; the enthalpy ceiling (also the one after
     * the arc injection, which reads the fields of the previous step), the
     * floor, the phase update, Marangoni and the remelt / trailing-freeze
     * tail use the fields; variable_tau replaces the collision by the
     * variable-tau SRT (solvers/coupled_step.py:168-458). */
    int use_tables, variable_tau;
    float rho_mat;          /* rho of the material [kg/m^3] */
    float force_scale_lu;   /* Marangoni prefactor force_scale / dx */
    float marangoni_scale;
    float H_sol_t, H_liq_t; /* rho * cp(T_solidus) * T_solidus, H_sol_t + L_rho */
    float tau_ref;          /* grid tau (SOLID / GAS cells) */
    WaamMaterialTables tables;
    /* pipelined stream: the stream of step n reads and writes only population
     * buffers, and step n + 1 touches them again only from its column pass on
     * (the collision writes the buffer the stream of step n writes), while
     * its arc, thermal and VOF stages only read the flags the stream reads.
     * defer_stream = 1: waam_step_main leaves this step's stream pending;
     * stream_prev = 1: it is pending from the step before -- waam_step_pre
     * starts it on a library stream beside the arc, thermal and VOF stages and
     * waam_step_main joins it before the column pass, or after it when the
     * stream reads the flag copies (WaamFields.flags_copy_r).  A caller that reads or
     * writes populations between steps runs the pending stream first with
     * waam_step_stream.  defer_stream needs the remelt / solidify tail off
     * (it writes flags after the stream). */
    int stream_prev;
    int defer_stream;
    /* pipelined collision: the collision of step n (with the tracers) needs
     * the column pass of step n, and step n + 1 needs its velocities only
     * from its thermal and VOF stages on, while its arc stage reads flags, f_l
     * and phi and writes H.  defer_collide = 1 (needs defer_stream = 1, no
     * force buffer, no collision tape, no Lorentz fields): waam_step_main
     * stops after the column pass and leaves collision, tracers and stream
     * pending; collide_prev = 1: they are pending from the step before
     * (welding flag collide_prev_welding) -- waam_step_pre runs the collision
     * beside the arc stage and the stream after it, and waam_step_main waits
     * for the collision before its thermal and VOF stages.  A caller that
     * reads populations, density, velocity, forces or tracers between steps
     * runs the pending work first with waam_step_finish. */
    int collide_prev;
    int collide_prev_welding;
    int defer_collide;
    /* shielding-gas shear and vapour recoil in the force assembly while
     * welding (physics/weld_forces.py:137-193): gas_shear on/off with the
     * peak shear stress; recoil 0 off, 1 T-ratio form (recoil_pa, recoil_T_ref),
     * 2 Clausius-Clapeyron form (P_ref, T_boil, L_vap, R_spec, C_acc); both
     * over the Gaussian of width weld_sigma (cells) around the torch */
    int gas_shear;
    float gs_tau_pa;
    int recoil;
    float recoil_pa, recoil_T_ref, P_ref, T_boil, L_vap, R_spec, C_acc, weld_sigma;
    /* density band of the health word's WAAM_HEALTH_RHO_RANGE bit (the check
     * is off when rho_hi <= rho_lo) */
    float rho_lo, rho_hi;
    /* quiet-tile skipping (needs WaamFields.tile_*): 1 skips the quiet tiles
     * of this step; 0 works every tile and restarts the tile history (the
     * step after a state change, a droplet deposition, a force clear, or
     * with the remelt / solidify tail on) */
    int tile_skip;
    /* lagged stream.  The collision of step n + 1 overwrites every population
     * of its active cells in the buffer the stream of step n writes, and
     * reads the buffer that stream reads, so the stream of step n needs to
     * visit only the other cells -- and then depends on neither the
     * collision of step n + 1 nor anything of step n + 1 but its column
     * pass.  hold_stream = 1 (needs stream_prev = 1, defer_collide = 1 and
     * the three flag copies): waam_step_pre does not run the previous step's
     * pending stream; it stays pending, and the next step runs it with
     * stream_lag = 1: waam_step_pre starts it at once beside the pending
     * collision (which must be pending: collide_prev = 1), skipping the cells
     * active in flags_copy_r, with the flags of flags_copy_rr; waam_step_main
     * joins it after the column pass.  waam_step_finish with stream_lag = 1
     * runs it before the pending collision. */
    int stream_lag;
    int hold_stream;
    /* 1: the collision takes the populations of the cells whose slot in
     * WaamFields.pop_cache_src holds their index and the previous step's
     * stamp from that slot.  Only when nothing but the fused step's own
     * collision and stream has written the populations since the previous
     * collision (not after a droplet deposition, a state load, the moving
     * window or an operator call). */
    int cache_read;
    /* cache_read of the pending collision (collide_prev = 1): the previous
     * step's own cache_read */
    int collide_prev_cache_read;
} WaamStepParams;

/* Stages of one fused step.  waam_step_pre runs the surface-height query,
 * the arc weight sum, the arc heat injection and the enthalpy cap
 * (solvers/coupled_step.py:34-108).  The host then performs droplet
 * deposition if one is due, and calls waam_step_main for the rest of the
 * step (coupled_step.py:168-458).  waam_step_main forks independent kernels
 * onto a second stream of the library's own (one per device, created on the
 * first call -- make that call outside any stream capture) and joins it back
 * into `stream` before returning; a capture of `stream` records the fork as
 * graph branches. */
int waam_step_pre(const WaamFields* f, const WaamStepParams* p, void* workspace,
                  size_t workspace_bytes, void* stream);
int waam_step_main(const WaamFields* f, const WaamStepParams* p, void* workspace,
                   size_t workspace_bytes, void* stream);
/* The stream left pending by the previous step (WaamStepParams.defer_stream),
 * for fields that describe the step after it (buffers swapped): reads f_src,
 * writes f_dst, with the flags of that step. */
int waam_step_stream(const WaamFields* f, const WaamStepParams* p, void* stream);
/* The collision, tracers and stream left pending by the previous step
 * (WaamStepParams.defer_collide; p->collide_prev_welding and
 * p->collide_prev_cache_read are that step's welding flag and cache_read),
 * for fields that describe the step after it (buffers
 * swapped, thermal fields flipped). */
int waam_step_finish(const WaamFields* f, const WaamStepParams* p, void* workspace,
                     size_t workspace_bytes, void* stream);
/* waam_step_main that also records events[0..6] (cudaEvent_t handles) on the
 * stream at the stage boundaries: before thermal, after thermal, after VOF
 * advection, after the column pass, after collide, after stream, after the
 * remelt/solidify tail (a skipped stage has zero duration). */
int waam_step_main_events(const WaamFields* f, const WaamStepParams* p, void* workspace,
                          size_t workspace_bytes, void* const* events, int n_events,
                          void* stream);

/* waam_step_main in two halves around the Lorentz solve, which reads the
 * liquid fraction and flags of this step and writes the J and B the
 * collision adds: stage 0 = VOF advection, thermal, phase, flags and the
 * active-cell list; stage 1 = forces, collision, stream, tracers, tail.
 * Stage 0 followed by stage 1 equals one waam_step_main.  events: null, or
 * the 7 handles of waam_step_main_events given to both calls (stage 0
 * records 0..3, stage 1 records 4..6). */
int waam_step_main_stage(const WaamFields* f, const WaamStepParams* p, int stage, void* workspace,
                         size_t workspace_bytes, void* const* events, int n_events,
                         void* stream);
/* Number of kernels the fused stages launch (for launch accounting): stage 0
 * waam_step_pre, 1 waam_step_main, 2 waam_step_main_events; the J x B pass
 * over SOLID cells of a step with WaamFields.lorentz_J set adds one).  f may
 * be null (then: without the quiet-tile buffers). */
int waam_step_launch_count(const WaamFields* f, const WaamStepParams* p, int stage);

/* ---- adjoint of the coupled step (reverse kernels, one step each) ---------- */
/* The reverse step runs: waam_adj_stream, waam_adj_collide, waam_adj_combine,
 * waam_adj_thermal, waam_adj_inject (see waam_solver_b200/adjoint.py).  All
 * are gathers (no floating-point atomics); parameter sums are FP64 in a fixed
 * order.  VOF, flags and the active set are the forward trajectory's. */

/* stream transposed: lam_yp (in lam Y', out lam Y' + S^T lam X'), lam_xn (out:
 * lam X' at SOLID cells, 0 elsewhere); flags of step n + 1 */
int waam_adj_stream(float* lam_yp, const float* lam_xp, float* lam_xn, const int32_t* flags,
                    int nx, int ny, int nz, void* stream);
/* forces + MRT collision + Mach / force clamps at the taped active cells
 * (WaamFields.tape_*), then the gather of the Marangoni T terms; ctb holds
 * 6 floats per tape slot, map one int per cell (all -1 on entry and exit) */
int waam_adj_collide(const WaamStepParams* p, const float* tape_f, const int32_t* tape_cells,
                     const int32_t* tape_count, int64_t tape_cap, const float* phi,
                     const float* T, const float* f_l, const int32_t* flags,
                     const float* scalars, float* lam_yp, float* lam_xn, float* lam_ux,
                     float* lam_uy, float* lam_uz, float* lam_fl, float* lam_T, float* ctb,
                     int32_t* map, int nx, int ny, int nz, void* stream);
/* lam_H += dT/dH lam_T + df_l/dH lam_f_l at H (step n + 1); lam_T = lam_f_l = 0 */
int waam_adj_combine(const WaamStepParams* p, float* lam_H, float* lam_T, float* lam_fl,
                     const float* H, const int32_t* flags, const float* phi, int64_t n,
                     void* stream);
/* thermal stage transposed: lam_H (step n + 1) -> lam_Hp (post-injection H of
 * step n); lam_T and the velocity adjoints accumulate step n's terms;
 * grad_hconv[0] += d/d h_conv (FP64).  mu: one float per cell of scratch. */
int waam_adj_thermal(const WaamStepParams* p, const float* lam_H, float* lam_Hp, float* mu,
                     float* lam_T, float* lam_ux, float* lam_uy, float* lam_uz, const float* Hp,
                     const float* T, const float* ux, const float* uy, const float* uz,
                     const int32_t* flags, int nx, int ny, int nz, double* grad_hconv,
                     void* workspace, size_t workspace_bytes, void* stream);
/* injection + ceiling transposed: lam_Hp -> lam_H (step n); sums[0..10] +=
 * A, B_{af, ar, b, c, sigma}, D_{af, ar, b, c, sigma} (FP64) */
int waam_adj_inject(const WaamStepParams* p, float* lam_H, const float* lam_Hp, const float* H,
                    const float* f_l, const int32_t* flags, const float* scalars, int nx, int ny,
                    int nz, double* sums, void* workspace, size_t workspace_bytes, void* stream);
/* lam[cells[t]] += vals[t] for t < count (in order) */
int waam_adj_scatter_add(float* lam, const int32_t* cells, const float* vals, int count,
                         void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
