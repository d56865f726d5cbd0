// bb_kernels.cuh -- host-side launchers of the step's kernels (one .cu file per stage).
#pragma once
#include "bb_common.cuh"

// bb_scan_sort.cu
// skip (device word, may be null): when non-zero the scan does nothing (not even its total)
void bb_launch_scan(cudaStream_t s, const uint32_t* in, uint32_t* out, const uint32_t* n_dev, uint32_t n_cap,
                    uint32_t* total, unsigned long long* status, uint32_t* tile_ctr, DevCounters* ctr,
                    const uint32_t* skip = nullptr);
uint32_t bb_scan_tiles(uint32_t n_cap);
uint32_t bb_sort_tiles(uint32_t n_cap);
void onesweep_smem_attr();  // k_onesweep's dynamic shared memory size, once per device
#define BB_SORT_TILE 8192  // keys per onesweep tile
// hist regions are BB_HIST_REGION words: 8 rows of counts + 8 rows of exclusive starts
#define BB_HIST_REGION (2 * 8 * 256)
void bb_launch_sort(cudaStream_t s, uint32_t* keys[2], uint32_t* vals[2], const uint32_t* n_dev, uint32_t n_cap,
                    int passes, int shift0, uint32_t* hist, uint32_t* status, uint32_t* tile_ctr, DevCounters* ctr,
                    int sms, const uint32_t* lut = nullptr, int lut_passes = 0);
void bb_launch_sort_to(cudaStream_t s, const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* dst_keys[2],
                       uint32_t* dst_vals[2], uint32_t n, int passes, uint32_t* hist, uint32_t* status,
                       uint32_t* tile_ctr, DevCounters* ctr, int sms);

// Scratch bookkeeping shared by the stages of one substep.
struct StepScratch {
  unsigned long long* scan_status;  // n_scans x scan_tiles
  uint32_t* scan_tile_ctr;          // n_scans
  uint32_t scan_tiles;
  uint32_t* sort_hist;              // n_sorts x (2 x 4 x 256)
  uint32_t* sort_status;            // n_sorts x 4 x sort_tiles x 256
  uint32_t* sort_tile_ctr;          // n_sorts x 4
  uint32_t sort_tiles;
};

// bb_bvh.cu: Morton codes -> sort -> Karras LBVH -> refit -> broad phase.  marks (may be
// null): four events recorded after the Morton codes, the sort, the tree build and the refit.
void bb_front_end(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc, int sms,
                  int cur, uint32_t max_world_bodies, cudaEvent_t* marks = nullptr);

// bb_narrow.cu: narrow phase + warm start + manifold compaction + per-body lists
void bb_narrow_phase(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc,
                     int sms, int cur, bool warm);

// bb_graph.cu: advect, islands, sleeping, edge colouring + colour buckets
void bb_advect(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, float h, int sms);
void bb_islands(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc, int sms,
                int cur, int coop_blocks);
int bb_components_blocks(int sms);
void bb_sleep(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, int sms, int cur);
void bb_edge_coloring(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc,
                      int sms, int cur, int coop_blocks);

// bb_solve.cu: PGS_SOFT and AVBD solvers
void bb_solve_islands(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, float h, int cur,
                      const StepScratch& sc, int sms);
void bb_solve_pgs_soft(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, float h, int cur,
                       const StepScratch& sc, int coop_blocks, int sms);
void bb_solve_avbd(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, float h, const StepScratch& sc,
                   int sms, int cur, int coop_blocks);

// serving loop helpers (bb_world.cu): one batch slot's state, the device error word
bb_status bb_world_read_range(void* world, uint32_t first, uint32_t count, float* position, float* rotation,
                              float* velocity, float* omega, uint32_t* flags);
const uint32_t* bb_world_error_word(void* world);

// thread-local last-error message behind bb_last_error_string (bb_world.cu)
bb_status bb_fail(bb_status code, const char* msg);

// stand-alone radix sort helpers (bb_sort_api.cu)
char* bb_sort_scratch_base();
bb_status bb_check_sort_args(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                             uint32_t n, uint32_t key_bits);
void bb_sort_carve(char* base, uint32_t n, int passes, DevCounters** ctr, uint32_t** hist, uint32_t** tile_ctr,
                   uint32_t** status, uint32_t** tmp_keys, uint32_t** tmp_vals, size_t* zero_bytes);

// co-resident block counts of the persistent cooperative kernels
int bb_edge_coloring_blocks(int sms);
int bb_pgs_soft_blocks(int sms);
int bb_avbd_blocks(int sms);

// occupancy helpers (bb_world.cu)
int bb_coop_blocks(const void* kernel, int threads, int sms);
cudaError_t bb_launch_coop(const void* kernel, int blocks, int threads, void** args, cudaStream_t s,
                           size_t smem_bytes = 0);
