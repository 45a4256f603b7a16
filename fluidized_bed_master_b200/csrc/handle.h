// handle.h -- host-side state of an engine handle (internal).
#pragma once
#include <cuda_runtime.h>
#include <map>
#include <string>
#include <vector>
#include "../../include/sphdem.h"

struct SphdemHandle {
    SphdemParams p;
    int ns = 0, nd = 0;
    int device = 0;
    int prec = SPHDEM_PREC_FP32;
    cudaStream_t stream = nullptr;
    bool committed = false;
    // staged host input (input order) until commit
    std::map<int, std::vector<double>> stage_d[2];
    std::map<int, std::vector<int>> stage_i[2];
    // rows in file order for the bounding box (SPH then DEM if set
    // programmatically; input.txt order if read from a directory)
    std::vector<double> file_x, file_y, file_z;
    double file_h0 = 0.0;
    bool have_file_order = false;
    double time = 0.0;
    int count = 0;
    double bbox[6] = {0, 0, 0, 0, 0, 0};
    int nijk[3] = {0, 0, 0};
    double dcell = 0.0;
    void* eng = nullptr;     // engine host state (EngineHost or WEngineHost, by kind)
    int kind = 0;            // 0 ISPH-DEM step, 1 2-D WCSPH step
    std::map<int, cudaGraphExec_t> graphs;
    std::map<int, int64_t> graph_launches;
    std::map<int, std::vector<int>> graph_kused;
    int use_graphs = 1;
    bool capturing = false;              // inside the capture of a step graph
    int mlp_phase = 0;                   // learned warm start of the step being built: 0 off, 1 train, 2 use
    cudaStream_t side = nullptr;         // captures the body of the PPE while node
    // DEM branch of the ISPH-DEM step: the DEM kernels that depend on no SPH
    // pass run on their own stream, forked from and joined to the step
    // stream by events (captured into the step graph as parallel branches)
    cudaStream_t dem_stream = nullptr;
    cudaEvent_t fork_ev[6] = {};
    int concurrent = 1;                  // sphdem_set_concurrency
    int time_only = -1;                  // sphdem_set_timing_only: the one kernel timed (-1 all)
    // the whole bed's domain for a slab of it (sphdem_set_domain, before commit)
    // per-bed open-boundary rows of a handle of 2-D beds (sphdem_set_beds),
    // sorted by plane; on the device as BED_COLS doubles per row
    std::vector<SphdemBedRow> beds;
    int list_build_req = 0;   // sphdem_set_list_build: 0 = tuned at commit
    double* d_beds = nullptr;
    bool dom_set = false;
    double dom_bbox[6] = {};
    double dom_h0 = 0, dom_tref = 0;
    // device scratch of the slab calls
    int* slab_blk = nullptr;             // per-block counts, then offsets
    int slab_blk_n = 0;
    int* slab_tot = nullptr;
    int* slab_free = nullptr;            // parked slots found by sphdem_slab_import
    int slab_free_n = 0;
    int64_t last_launches = 0;
    // per-kernel timing (events recorded inside the step graph)
    int timing = 0;
    std::vector<cudaEvent_t> ev_beg, ev_end;
    std::vector<int> ev_used;
    std::vector<double> kern_ms;
    std::vector<int64_t> kern_n;
    // device staging buffer of the bulk field transfers (doubles)
    double* xfer = nullptr;
    size_t xfer_elems = 0;
    int ppe_iters = 0;
    double ppe_res = 0.0;
    double ppe_ms = 0.0;
    // batch of independent 2-D beds in one handle (sphdem_create_batch):
    // rows bed_start[b] .. bed_start[b+1]-1 of the input are bed b, placed
    // at commit with its x, y shifted by bed_off[2b], bed_off[2b+1]
    std::vector<int> bed_start;
    std::vector<double> bed_off;
    // asynchronous output (sphdem_snapshot): the VTK fields packed into a
    // device buffer on the step stream, copied to pinned host memory on a
    // second stream; one entry per packed field
    struct SnapField {
        int which, field, kind;   // kind: 0 double, 1 R, 2 int32
        size_t off, bytes;
    };
    std::vector<SnapField> snap_fields;
    unsigned char* snap_dev = nullptr;
    unsigned char* snap_host = nullptr;
    size_t snap_bytes = 0;
    cudaStream_t snap_stream = nullptr;
    cudaEvent_t snap_packed = nullptr, snap_done = nullptr;
    bool snap_pending = false;
    double snap_t_ref = 0.0;      // offset of the SPH temperature at the snapshot
    int snap_count = 0;
    double snap_time = 0.0;
};

// io.cpp
int sphdem_io_read_input_txt(const char* path, SphdemHandle* h, const SphdemParams* p);
int sphdem_io_check_table(const char* path);
void sphdem_io_params_default(SphdemParams* p);
int sphdem_io_write_vtk_dem(const char* path, int n, const double* x, const double* y, const double* z,
                            const int* itype, const int* ptype, const int* dem_idx, const double* magf,
                            const double* eliz, const double* por, const double* uz, const double* qsd,
                            const double* ftz, const double* temp, const double* rad, const double* dtemp);
// fluid particles (p_type 1) of the SPH set in the layout of
// save_plot_fluid_vtk_bin_fluid_sph (functions_OUTPUT.cuh:445-651)
int sphdem_io_write_vtk_fluid(const char* path, int n, const int* ptype, const double* x, const double* y,
                              const double* z, const double* por, const double* pres, const double* dtemp,
                              const int* btype, const double* rho, const double* temp, const double* uz);
