/* zebsdsolve.h — the reference's own C ABI (zebsdsolve 0.2.8), as libzebsdsolve.so exports it.
 *
 * These are the calls of src/exports.zig and src/native_api.zig, with their argument types and
 * extern-struct layouts, which python/zebsdsolve/_native.py:95-174 binds through ctypes (77 of them;
 * ze_cell_info, ze_cell_view, ze_sim_energy and ze_sphere_view are the web module's). The library
 * carries each call out on this package's engine (zebsdsolve_b200/ze_abi.py) and its sm_100a kernels
 * (libzebsdsolve_b200.so, include/zebsdsolve_b200.h), so the reference's Python package runs over it
 * unmodified:
 *
 *     ZEBSDSOLVE_LIB=<package>/libzebsdsolve.so ZEBSDSOLVE_WGPU=<any path> python ...
 *
 * Conventions (exports.zig:1-8): 0, a count, size or index on success; a negative code on failure,
 * ze_error() then saying why (and clearing it). A call that fills a buffer returns the size it needs
 * and copies only when the capacity given suffices. The handle from ze_create is opaque; the adapter
 * path it takes is not used (the engine runs on the current CUDA device).
 *
 * Not part of this engine (the call fails, ze_error says so): master simulation and crystals
 * (ze_sim_*, ze_cell_info, ze_cell_view, ze_sphere_view), the IPF
 * colours (ze_map's kinds 0-2, ze_ipf_key; its score, phase and sweep maps, kinds 3-7, are built),
 * the .h5oina export, WGSL (ze_compile_wgsl reports that none is compiled; ze_shader lists no
 * modules).
 *
 * A native host (not a Python process) links libpython3.12 as well; the first call then starts an
 * interpreter, which finds the package beside the library.
 */
#ifndef ZEBSDSOLVE_H
#define ZEBSDSOLVE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* engine.zig:55-75 */
typedef struct {
  uint32_t rows, cols, pat_h, pat_w;
  uint32_t pixel; /* 0 u8, 1 u16, 2 f32 */
  uint32_t has_background, has_pc;
  uint32_t format; /* scan.zig:27 Format's index; 100: patterns from memory */
  double voltage_kv, bytes;
  uint32_t has_px, pattern_kinds;
} ze_ScanInfo;

/* engine.zig:77-89 */
typedef struct {
  uint32_t side, point_group, space_group, laue;
  uint32_t n_fold, mirror, inversion, pad;
  double voltage_kv;
  char name[64];
} ze_PhaseInfo;

/* geometry.zig:28-50 */
typedef struct {
  double pc[3];
  double sample_tilt_deg, detector_tilt_deg;
  double rot[3];
  double px_um, step_x_um, step_y_um;
  uint32_t plane_kind, pad;
  double plane[12];
} ze_Geometry;

/* pcfit.zig Result */
typedef struct {
  double pc[3], start[3];
  double score, start_score;
  uint32_t n_patterns, n_candidates, levels, at_border;
} ze_PcResult;

/* planefit.zig PlaneResult */
typedef struct {
  double plane[12], pc[3], start_pc[3], rot[3];
  double said_rot[3], said_rot_se[3], step[2], step_se[2], skew, skew_se;
  double pc_se[3], rmsd[3], ncc, start_ncc;
  uint32_t kind, frame, n_patterns, n_used, iterations, blocks, model, compared;
  double cv[4], cv_se[4];
  uint32_t method, pad;
} ze_PlaneResult;

/* planefit.zig PlanePoint */
typedef struct {
  uint64_t cell;
  double pc[3], fit[3], ncc;
  uint32_t used, pad;
} ze_PlanePoint;

/* simulate.zig Summary */
typedef struct {
  uint32_t n_k, n_sites, n_g, n_bins, n_bins_run, max_beams;
  uint32_t failed, stopped, halfw, rank, max_weak, overflow;
  double last_change;
} ze_SimSummary;

/* engine.zig:92-107 */
typedef struct {
  uint32_t sweep, sweeps, bandwidth, dict_grid;
  uint64_t done, total, region, accepted;
  uint32_t method, pad;
} ze_IndexStatus;

/* creation: native_api.zig:18, 24, 39, 45 */
const char* ze_version(void);
void* ze_create(const char* lib_path);
size_t ze_create_error(char* buf, size_t cap);
void ze_destroy(void* e);

/* plumbing: exports.zig:30, 38, 43, 50, 58, 63 */
size_t ze_adapter(void* e, char* buf, size_t cap);
size_t ze_error(void* e, char* buf, size_t cap);
int32_t ze_configure(void* e, const char* json, size_t len);
size_t ze_settings(void* e, char* buf, size_t cap);
size_t ze_events(void* e, char* buf, size_t cap);
void ze_cancel(void* e);

/* scan: exports.zig:70, 85, 97, 104, 108, 113, 453, 459, 823 */
int32_t ze_open_scan(void* e, const char* paths, size_t len);
int32_t ze_set_patterns(void* e, const void* data, size_t len, uint32_t pixel, uint32_t rows, uint32_t cols,
                        uint32_t h, uint32_t w);
int32_t ze_synthesize(void* e, float* quats, int32_t* phase, int32_t* grain, size_t n);
void ze_close_scan(void* e);
void ze_scan_info(void* e, ze_ScanInfo* out);
size_t ze_scan_format(void* e, char* buf, size_t cap);
uint32_t ze_scan_overview_kind(void* e);
int64_t ze_scan_overview(void* e, float* out, size_t cap);
int32_t ze_stored_orientations(void* e, double* euler, int32_t* phase, uint64_t n);

/* geometry: exports.zig:124, 141 */
void ze_get_geometry(void* e, ze_Geometry* out);
void ze_set_geometry(void* e, const ze_Geometry* in);

/* phases: exports.zig:160, 365, 369, 373, 393 */
int32_t ze_add_phase(void* e, const char* path, size_t len);
void ze_clear_phases(void* e);
uint32_t ze_phase_count(void* e);
int32_t ze_phase_info(void* e, uint32_t index, ze_PhaseInfo* out);
int32_t ze_master_image(void* e, uint32_t phase, float* out, size_t len);

/* master simulation: exports.zig:174, 204, 230, 284, 294, 306, 314, 324, 336, 345, 357, 386 */
int32_t ze_sim_read_cif(void* e, const char* text, size_t len);
int32_t ze_sim_set_crystal(void* e, const char* json, size_t len);
int32_t ze_sim_edit_crystal(void* e, const char* json, size_t len);
int64_t ze_sim_crystal(void* e, void* out, size_t cap);
int64_t ze_cell_info(void* e, uint32_t cells, void* out, size_t cap);
int32_t ze_cell_view(void* e, const float* view_rot, float zoom, uint32_t highlight, uint32_t cells, uint32_t width,
                     uint32_t height, uint32_t* out, size_t len);
int64_t ze_sim_energy(void* e, void* out, size_t cap);
int32_t ze_sim_run(void* e, ze_SimSummary* out);
int32_t ze_sim_sheets(void* e, float* out, size_t cap);
int32_t ze_sim_add_phase(void* e, const char* name, size_t len);
int64_t ze_sim_npz(void* e, void* out, size_t cap);
int32_t ze_sphere_view(void* e, int32_t source, uint32_t stored, int32_t bin, int32_t site, uint32_t projection,
                       const float* view_rot, float zoom, uint32_t width, uint32_t height, uint32_t* out, size_t len);

/* patterns: exports.zig:401, 411, 423, 433, 442, 447, 470 */
int32_t ze_pattern_shape(void* e, uint32_t full, uint32_t* out);
int32_t ze_pattern(void* e, uint64_t cell, uint32_t processed, uint32_t full, float* out, size_t len);
uint32_t ze_nlpar_view(void* e, float* out, float* shares, size_t cap);
int64_t ze_lattice(void* e, uint32_t want, uint64_t* out, size_t cap);
double ze_pixel_angle(void* e);
int32_t ze_pattern_stats(void* e, const uint64_t* cells, size_t n, float* out, size_t len);
int32_t ze_simulate(void* e, uint32_t phase, const uint64_t* cells, const float* quats, size_t n, uint32_t full,
                    float* out, size_t len);

/* fits: exports.zig:478, 486, 502, 511, 533, 545, 555, 563, 570, 580 */
int32_t ze_fit_pc(void* e, ze_PcResult* out);
int32_t ze_pc_scores(void* e, uint32_t* shape, double* axes, size_t axes_cap, float* scores, size_t cap);
uint32_t ze_pc_level_count(void* e);
int32_t ze_pc_level(void* e, uint32_t i, uint32_t* shape, uint32_t* info, double* axes, size_t axes_cap,
                    float* scores, size_t cap, uint32_t* pat_best, float* pat_ncc, size_t pat_cap);
int32_t ze_pc_level_scores(void* e, uint32_t i, float* out, size_t cap);
int32_t ze_pc_level_ballots(void* e, uint32_t i, float* out, size_t cap, double* info);
int32_t ze_fit_auto(void* e, ze_PlaneResult* out);
int32_t ze_fit_plane(void* e, ze_PlaneResult* out);
size_t ze_plane_points(void* e, ze_PlanePoint* out, size_t cap);
int32_t ze_fit_patterns(void* e, uint64_t* cells, int32_t* phases, float* quats, float* ncc, size_t cap);

/* indexing: exports.zig:594, 603, 613, 618, 623, 631, 638, 644, 653, 666, 679, 693 */
int32_t ze_index_begin(void* e);
int64_t ze_index_step(void* e);
int32_t ze_tune_begin(void* e);
int32_t ze_tune_trial(void* e);
int32_t ze_tune_report(void* e, double seconds);
int32_t ze_chance(void* e, uint32_t phase, float* out);
void ze_index_status(void* e, ze_IndexStatus* out);
void ze_sweep(void* e, uint32_t i, uint32_t* out);
int32_t ze_index_cells(void* e, const uint64_t* cells, size_t n, float* out, size_t len);
int32_t ze_cell_under(void* e, uint64_t cell, const ze_Geometry* geo, uint32_t bandwidth, uint32_t full, float* recs,
                      size_t n_recs, float* sim, size_t len);
int32_t ze_index_cells_by(void* e, const uint64_t* cells, size_t n, uint32_t method, uint32_t bandwidth,
                          uint32_t dict_grid, float* out, size_t len);
int64_t ze_results(void* e, uint32_t kind, void* out, size_t len);

/* results out: exports.zig:726, 739, 748, 758, 789, 838, 849, 865, 874 */
int32_t ze_map(void* e, uint32_t kind, uint8_t* out, size_t len);
int32_t ze_ipf_key(void* e, uint32_t phase, uint32_t size, uint32_t lower, uint8_t* out, size_t len, float* box);
int64_t ze_export(void* e, uint32_t kind, void* buf, size_t cap);
int64_t ze_export_h5oina(void* e, void* buf, size_t cap);
int64_t ze_identify_frame(void* e, const double* euler, const int32_t* phase, uint64_t n, char* buf, size_t cap);
size_t ze_frame(void* e, char* buf, size_t cap);
int32_t ze_set_frame(void* e, const char* json, size_t len);
void ze_reduce(void* e, uint32_t phase, float* q, double* euler);
double ze_disorientation(void* e, uint32_t phase, const float* a, const float* b);

/* tests and profiling: exports.zig:883, 901, 918, 924, 929 */
int32_t ze_compile_wgsl(void* e, const char* code, size_t code_len, const char* entry, size_t entry_len, char* msg,
                        size_t cap);
size_t ze_shader(uint32_t index, char* name, size_t name_cap, void* buf, size_t cap);
void ze_gpu_counts(void* e, uint32_t* out);
int32_t ze_profile(void* e, uint32_t on);
size_t ze_profile_report(void* e, char* buf, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* ZEBSDSOLVE_H */
