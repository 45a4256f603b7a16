// ref_harness.cu -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference (SOPHIA_gpu.cu and the headers it includes, read
// unchanged from REF_DIR via -I) into a shared library and drives its own
// step function SOPHIA_single_ISPH (ISPH_Calc_seperate.cuh:13-503) on a
// GPU, and the 2-D WCSPH kernels of SOPHIA_single (WCSPH_Calc.cuh:15-340)
// in the Lagrangian order described at ref_load_wcsph.  The set-up below repeats what ISPH() (ISPH.cuh:10-200) and
// ISPH_Calc() (ISPH_Calc_seperate.cuh:508-903) do for one GPU, without the
// pthread fan-out and without the run-to-time_end loop, so that the state
// can be read back after a chosen number of steps.  Used only to generate
// golden fixtures (tests/golden/make_golden.py) and reference timings.
//
// Particle identity: the harness stores the input row of every SPH
// particle in part1::concn, which the ISPH step never reads or writes
// while Concentration-diffusion is NO; DEM particles carry dem_idx.
#include <unistd.h>
#include <chrono>
// wall-clock helper defined before the reference's macros (count, time, ...)
static std::chrono::steady_clock::time_point refh_now() { return std::chrono::steady_clock::now(); }
static double refh_ms(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

#define main sophia_reference_main
#include "SOPHIA_gpu.cu"
#undef main

namespace refh {
int_t *g_idx, *p_idx, *g_idx_in, *p_idx_in, *g_str, *g_end;
int_t *g_idx_sph, *p_idx_sph, *g_idx_sph_in, *p_idx_sph_in, *g_str_sph, *g_end_sph;
int_t *g_idx_dem, *p_idx_dem, *g_idx_dem_in, *p_idx_dem_in, *g_str_dem, *g_end_dem;
part1 *dP1, *dSP1, *dP1s, *dSP1s, *dP1d, *dSP1d;
part2 *dP2, *dSP2, *dP2s, *dSP2s, *dP2d, *dSP2d;
part3 *dP3, *dP3s, *dP3d;
int *aps_num_part, *aps;
void *st_all, *st_sph, *st_dem;
size_t sb_all, sb_sph, sb_dem;
part1 *fP1, *fP1s, *fP1d;
part2 *fP2, *fP2s, *fP2d;
part3 *fP3, *fP3s, *fP3d;
Real dummy[16];
int loaded = 0;
double last_ms = 0.0;
}  // namespace refh

using namespace refh;

#define HCK(call)                                   \
    do {                                            \
        if ((call) != cudaSuccess) return -100;     \
    } while (0)

// want: Isph (SOPHIA_single_ISPH) or Wcsph (the 2-D SOPHIA_single below)
static int load_impl(const char* workdir, int want) {
    if (chdir(workdir) != 0) return -1;
    memset(vii, 0, sizeof(int_t) * vii_size);
    memset(vif, 0, sizeof(Real) * vif_size);
    ngpu = 1;
    read_solv_input(vii, vif, "./input/solv.txt");
    read_table("./input/data.txt");
    if (solver_type != want) return -2;
    if (want == Wcsph && dim != 2) return -3;
    // ISPH.cuh:55-120
    num_part = gpu_count_particle_numbers2("./input/input.txt");
    HP1 = (part1*)malloc(num_part * sizeof(part1));
    memset(HP1, 0, sizeof(part1) * num_part);
    read_input(HP1);
    num_part_sph = gpu_count_particle_numbers_sph(HP1);
    num_part_dem = gpu_count_particle_numbers_dem(HP1);
    HP1_sph = (part1*)malloc(num_part_sph * sizeof(part1));
    HP1_dem = (part1*)malloc(num_part_dem * sizeof(part1));
    memset(HP1_sph, 0, sizeof(part1) * num_part_sph);
    memset(HP1_dem, 0, sizeof(part1) * num_part_dem);
    read_sph_dem(HP1, HP1_sph, HP1_dem);
    for (int k = 0; k < num_part_sph; k++) HP1_sph[k].concn = (Real)k;   // identity tag
    if (want == Wcsph) {
        if (num_part_dem != 0) return -4;
        for (int k = 0; k < num_part; k++) HP1[k].concn = (Real)k;
    }
    Real cell_reduction_factor = 1.1;
    search_incr_factor = 1.0;
    search_kappa = kappa;
    find_minmax(vii, vif, HP1);
    Real h0 = HP1[0].h;
    dcell = cell_reduction_factor * kappa * h0;
    NI = (int)((x_max - x_min) / dcell) + 1;
    NJ = (int)((y_max - y_min) / dcell) + 1;
    NK = (int)((z_max - z_min) / dcell) + 1;
    calc_area = ceil(NI / ngpu);
    num_part2 = num_part;
    num_part2_sph = num_part_sph;
    num_part2_dem = num_part_dem;
    pthread_barrier_init(&barrier, NULL, 1);
    // ISPH_Calc_seperate.cuh:516-903 for tid 0
    num_cells = clc_num_cells();
    count = floor(time / dt + 0.5);
    HCK(cudaSetDevice(0));
    cudaStreamCreate(&str1[0]);
    cudaStreamCreate(&str2[0]);
    fP1 = (part1*)calloc(num_part2, sizeof(part1));
    fP1s = (part1*)calloc(num_part2_sph, sizeof(part1));
    fP1d = (part1*)calloc(num_part2_dem ? num_part2_dem : 1, sizeof(part1));
    fP2 = (part2*)calloc(num_part2, sizeof(part2));
    fP2s = (part2*)calloc(num_part2_sph, sizeof(part2));
    fP2d = (part2*)calloc(num_part2_dem ? num_part2_dem : 1, sizeof(part2));
    fP3 = (part3*)calloc(num_part2, sizeof(part3));
    fP3s = (part3*)calloc(num_part2_sph, sizeof(part3));
    fP3d = (part3*)calloc(num_part2_dem ? num_part2_dem : 1, sizeof(part3));
    HCK(cudaMalloc((void**)&aps_num_part, sizeof(int)));
    HCK(cudaMalloc((void**)&aps, sizeof(int)));
#define AL(p, T, n) HCK(cudaMalloc((void**)&p, sizeof(T) * ((n) ? (n) : 1)))
    AL(g_idx, int_t, num_part2); AL(p_idx, int_t, num_part2); AL(g_idx_in, int_t, num_part2);
    AL(p_idx_in, int_t, num_part2); AL(g_str, int_t, num_cells); AL(g_end, int_t, num_cells);
    AL(g_idx_sph, int_t, num_part2_sph); AL(p_idx_sph, int_t, num_part2_sph);
    AL(g_idx_sph_in, int_t, num_part2_sph); AL(p_idx_sph_in, int_t, num_part2_sph);
    AL(g_str_sph, int_t, num_cells); AL(g_end_sph, int_t, num_cells);
    AL(g_idx_dem, int_t, num_part2_dem); AL(p_idx_dem, int_t, num_part2_dem);
    AL(g_idx_dem_in, int_t, num_part2_dem); AL(p_idx_dem_in, int_t, num_part2_dem);
    AL(g_str_dem, int_t, num_cells); AL(g_end_dem, int_t, num_cells);
    AL(dP1, part1, num_part2); AL(dSP1, part1, num_part2); AL(dP2, part2, num_part2);
    AL(dSP2, part2, num_part2); AL(dP3, part3, num_part2);
    AL(dP1s, part1, num_part2_sph); AL(dSP1s, part1, num_part2_sph); AL(dP2s, part2, num_part2_sph);
    AL(dSP2s, part2, num_part2_sph); AL(dP3s, part3, num_part2_sph);
    AL(dP1d, part1, num_part2_dem); AL(dSP1d, part1, num_part2_dem); AL(dP2d, part2, num_part2_dem);
    AL(dSP2d, part2, num_part2_dem); AL(dP3d, part3, num_part2_dem);
#undef AL
    cudaMemset(g_str, cu_memset, sizeof(int_t) * num_cells);
    cudaMemset(g_end, 0, sizeof(int_t) * num_cells);
    cudaMemset(g_str_sph, cu_memset, sizeof(int_t) * num_cells);
    cudaMemset(g_end_sph, 0, sizeof(int_t) * num_cells);
    cudaMemset(g_str_dem, cu_memset, sizeof(int_t) * num_cells);
    cudaMemset(g_end_dem, 0, sizeof(int_t) * num_cells);
    cudaMemset(dP1, 0, sizeof(part1) * num_part2); cudaMemset(dSP1, 0, sizeof(part1) * num_part2);
    cudaMemset(dP2, 0, sizeof(part2) * num_part2); cudaMemset(dSP2, 0, sizeof(part2) * num_part2);
    cudaMemset(dP3, 0, sizeof(part3) * num_part2);
    cudaMemset(dP1s, 0, sizeof(part1) * num_part2_sph); cudaMemset(dSP1s, 0, sizeof(part1) * num_part2_sph);
    cudaMemset(dP2s, 0, sizeof(part2) * num_part2_sph); cudaMemset(dSP2s, 0, sizeof(part2) * num_part2_sph);
    cudaMemset(dP3s, 0, sizeof(part3) * num_part2_sph);
    if (num_part2_dem) {
        cudaMemset(dP1d, 0, sizeof(part1) * num_part2_dem); cudaMemset(dSP1d, 0, sizeof(part1) * num_part2_dem);
        cudaMemset(dP2d, 0, sizeof(part2) * num_part2_dem); cudaMemset(dSP2d, 0, sizeof(part2) * num_part2_dem);
        cudaMemset(dP3d, 0, sizeof(part3) * num_part2_dem);
    }
    cudaMemcpyToSymbol(k_vii, vii, sizeof(int_t) * vii_size);
    cudaMemcpyToSymbol(k_vif, vif, sizeof(Real) * vif_size);
    cudaMemcpyToSymbol(k_Tab_T, host_Tab_T, sizeof(Real) * table_size);
    cudaMemcpyToSymbol(k_Tab_h, host_Tab_h, sizeof(Real) * table_size);
    cudaMemcpyToSymbol(k_Tab_k, host_Tab_k, sizeof(Real) * table_size);
    cudaMemcpyToSymbol(k_Tab_vis, host_Tab_vis, sizeof(Real) * table_size);
    cudaMemcpyToSymbol(k_table_index, host_table_index, sizeof(int) * 10);
    cudaMemcpyToSymbol(k_table_size, host_table_size, sizeof(int) * 10);
    DHP1[0] = (part1*)calloc(num_part2, sizeof(part1));
    DHP1_sph[0] = (part1*)calloc(num_part2_sph, sizeof(part1));
    DHP1_dem[0] = (part1*)calloc(num_part2_dem ? num_part2_dem : 1, sizeof(part1));
    for (int k = 0; k < num_part2; k++) DHP1[0][k].i_type = 3;
    for (int k = 0; k < num_part2_sph; k++) DHP1_sph[0][k].i_type = 3;
    for (int k = 0; k < num_part2_dem; k++) DHP1_dem[0][k].i_type = 3;
    c_initial_inner_outer_particle_single(HP1, DHP1[0], 0);
    if (want == Wcsph)   // Lagrangian: ALE flags 1 (KERNEL_set_alpha is not launched)
        for (int k = 0; k < num_part2; k++) DHP1[0][k].elix = DHP1[0][k].eliy = DHP1[0][k].eliz = 1.0;
    c_initial_inner_outer_particle_single_sph(HP1_sph, DHP1_sph[0], 0);
    c_initial_inner_outer_particle_single_dem(HP1_dem, DHP1_dem[0], 0);
    HCK(cudaMemcpy(dP1, DHP1[0], num_part2 * sizeof(part1), cudaMemcpyHostToDevice));
    HCK(cudaMemcpy(dP1s, DHP1_sph[0], num_part2_sph * sizeof(part1), cudaMemcpyHostToDevice));
    if (num_part2_dem) HCK(cudaMemcpy(dP1d, DHP1_dem[0], num_part2_dem * sizeof(part1), cudaMemcpyHostToDevice));
    st_all = st_sph = st_dem = NULL;
    sb_all = sb_sph = sb_dem = 0;
    cub::DeviceRadixSort::SortPairs(st_all, sb_all, g_idx_in, g_idx, p_idx_in, p_idx, num_part2);
    cub::DeviceRadixSort::SortPairs(st_sph, sb_sph, g_idx_sph_in, g_idx_sph, p_idx_sph_in, p_idx_sph, num_part2_sph);
    cub::DeviceRadixSort::SortPairs(st_dem, sb_dem, g_idx_dem_in, g_idx_dem, p_idx_dem_in, p_idx_dem, num_part2_dem);
    HCK(cudaDeviceSynchronize());
    HCK(cudaMalloc(&st_all, sb_all ? sb_all : 16));
    HCK(cudaMalloc(&st_sph, sb_sph ? sb_sph : 16));
    HCK(cudaMalloc(&st_dem, sb_dem ? sb_dem : 16));
    loaded = want == Wcsph ? 2 : 1;
    return 0;
}

extern "C" int ref_load(const char* workdir) { return load_impl(workdir, Isph); }

// 2-D WCSPH: SOPHIA_single (WCSPH_Calc.cuh:15-340) for a Lagrangian fluid.
// The stock driver makes SPH Eulerian (KERNEL_set_alpha), sorts only at
// count 0 and does not launch KERNEL_interaction2D (WCSPH_Calc.cuh:187), so
// no particle moves.  This driver launches the same kernels in the same
// order with ALE flags 1 (set at load), NNPS every step (the count == 0
// branch) and KERNEL_interaction2D(1, ...) at the place of the disabled line.
extern "C" int ref_load_wcsph(const char* workdir) { return load_impl(workdir, Wcsph); }

static void wcsph2d_step() {
    dim3 b, t;
    t.x = 128;
    int s = sizeof(int) * (t.x + 1);
    b.x = (num_part2 - 1) / t.x + 1;
    if (time_type == Pre_Cor) KERNEL_clc_predictor<<<b, t>>>(dt, time, dP1, dP2, dP3);
    cudaMemset(g_str, cu_memset, sizeof(int_t) * num_cells);
    KERNEL_index_particle_to_cell<<<b, t>>>(g_idx_in, p_idx_in, dP1);
    cub::DeviceRadixSort::SortPairs(st_all, sb_all, g_idx_in, g_idx, p_idx_in, p_idx, num_part2);
    KERNEL_reorder<<<b, t, s>>>(g_idx, p_idx, g_str, g_end, dP1, dP2, dSP1, dSP2);
    cudaMemset(dP3, 0, sizeof(part3) * num_part2);
    cudaMemcpy(dP1, dSP1, sizeof(part1) * num_part2, cudaMemcpyDeviceToDevice);
    KERNEL_clc_mass_update<<<b, t>>>(g_str, g_end, dSP1, dSP2, count);
    if ((kgc_solve > 0) || (delSPH_solve == Antuono)) gradient_correction(g_str, g_end, dSP1, dP3);
    KERNEL_clc_prep2D_coupling<<<b, t>>>(g_str, g_end, dSP1, count);
    KERNEL_clc_prep2D<<<b, t>>>(g_str, g_end, dSP1, dSP2, dP3, count);
    if (rho_type == Mass_Sum) KERNEL_clc_mass_sum_norm2D<<<b, t>>>(g_str, g_end, dSP1, dSP2);
    else KERNEL_clc_continuity_norm2D<<<b, t>>>(g_str, g_end, dSP1, dSP2, dP3);
    KERNEL_EOS<<<b, t>>>(dSP1, dSP2);
    KERNEL_interaction2D<<<b, t>>>(1, g_str, g_end, dSP1, dSP2, dP3);
    KERNEL_time_update_single<<<b, t>>>(dt, dSP1, dP1, dSP2, dP2, dP3, time, count);
    KERNEL_open_boundary_extrapolation3D_1<<<b, t>>>(time, g_str, g_end, dP1, dSP2, dP3, count, dt);
    if (xsph_solve) KERNEL_xsph2D<<<b, t>>>(1, g_str, g_end, dt, time, dSP1, dP1, dSP2);
}

extern "C" int ref_run_wcsph(int nsteps) {
    if (loaded != 2) return -1;
    cudaDeviceSynchronize();
    auto t0 = refh_now();
    for (int k = 0; k < nsteps; k++) {
        wcsph2d_step();
        time += dt;
        count++;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return -100;
    auto t1 = refh_now();
    last_ms = refh_ms(t0, t1);
    if (cudaGetLastError() != cudaSuccess) return -101;
    // state after the step: dev_P1 (part1), dev_SP2 (part2), dev_P3 (part3),
    // read back through the SPH slots of ref_get
    HCK(cudaMemcpy(fP1s, dP1, num_part2 * sizeof(part1), cudaMemcpyDeviceToHost));
    HCK(cudaMemcpy(fP2s, dSP2, num_part2 * sizeof(part2), cudaMemcpyDeviceToHost));
    HCK(cudaMemcpy(fP3s, dP3, num_part2 * sizeof(part3), cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int ref_run(int nsteps) {
    if (loaded != 1) return -1;
    cudaDeviceSynchronize();
    auto t0 = refh_now();
    for (int k = 0; k < nsteps; k++) {
        SOPHIA_single_ISPH(g_idx, p_idx, g_idx_in, p_idx_in, g_str, g_end, dP1, dSP1, dP2, dSP2, dP3, NULL, NULL,
                           NULL, NULL, st_all, &sb_all, fP1, fP2, fP3, 0, aps_num_part, aps, dummy, dummy, dummy,
                           dummy, dummy, dummy, g_idx_sph, p_idx_sph, g_idx_sph_in, p_idx_sph_in, g_str_sph,
                           g_end_sph, dP1s, dSP1s, dP2s, dSP2s, dP3s, st_sph, &sb_sph, g_idx_dem, p_idx_dem,
                           g_idx_dem_in, p_idx_dem_in, g_str_dem, g_end_dem, dP1d, dSP1d, dP2d, dSP2d, dP3d, st_dem,
                           &sb_dem, fP1s, fP2s, fP3s, fP1d, fP2d, fP3d);
        time += dt;   // ISPH_Calc_seperate.cuh:924-925
        count++;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return -100;
    auto t1 = refh_now();
    last_ms = refh_ms(t0, t1);
    if (cudaGetLastError() != cudaSuccess) return -101;
    // state after the step: dev_P1 (part1), dev_SP2 (part2), dev_P3 (part3)
    HCK(cudaMemcpy(fP1s, dP1s, num_part2_sph * sizeof(part1), cudaMemcpyDeviceToHost));
    HCK(cudaMemcpy(fP2s, dSP2s, num_part2_sph * sizeof(part2), cudaMemcpyDeviceToHost));
    HCK(cudaMemcpy(fP3s, dP3s, num_part2_sph * sizeof(part3), cudaMemcpyDeviceToHost));
    if (num_part2_dem) {
        HCK(cudaMemcpy(fP1d, dP1d, num_part2_dem * sizeof(part1), cudaMemcpyDeviceToHost));
        HCK(cudaMemcpy(fP2d, dSP2d, num_part2_dem * sizeof(part2), cudaMemcpyDeviceToHost));
        HCK(cudaMemcpy(fP3d, dP3d, num_part2_dem * sizeof(part3), cudaMemcpyDeviceToHost));
    }
    return 0;
}

// SOPHIA_single_ISPH (ISPH_Calc_seperate.cuh:44-466) for decouple_stride 1,
// launch for launch, without the three DEM wall kernels (KERNEL_treat_DEM_
// {cylinder_z,box_z,truncated_cone_z}_dem), whose wall geometry the
// reference hard-wires (functions_DEM_BC.cuh): beds of another shape (the
// box bed) are timed with it.  The VTK output branch is left out as well
// (freq_output is set beyond the run).  Each step ends with a device sync,
// as the reference's does.
static void isph_step_without_dem_walls() {
    dim3 b, t;
    t.x = 128;
    int s = sizeof(int) * (t.x + 1);
    const int bs = (num_part2_sph - 1) / t.x + 1, bd = (num_part2_dem - 1) / t.x + 1;
    b.x = bs; KERNEL_set_alpha_sph<<<b, t>>>(dP1s);
    b.x = bd; KERNEL_set_alpha_dem<<<b, t>>>(dP1d);
    cudaDeviceSynchronize();
    cudaMemset(g_str_sph, cu_memset, sizeof(int_t) * num_cells);
    cudaMemset(g_str_dem, cu_memset, sizeof(int_t) * num_cells);
    cudaDeviceSynchronize();
    b.x = bs; KERNEL_index_particle_to_cell_sph<<<b, t>>>(g_idx_sph_in, p_idx_sph_in, dP1s);
    b.x = bd; KERNEL_index_particle_to_cell_dem<<<b, t>>>(g_idx_dem_in, p_idx_dem_in, dP1d);
    cudaDeviceSynchronize();
    cub::DeviceRadixSort::SortPairs(st_sph, sb_sph, g_idx_sph_in, g_idx_sph, p_idx_sph_in, p_idx_sph, num_part2_sph);
    cub::DeviceRadixSort::SortPairs(st_dem, sb_dem, g_idx_dem_in, g_idx_dem, p_idx_dem_in, p_idx_dem, num_part2_dem);
    cudaDeviceSynchronize();
    b.x = bs; KERNEL_reorder_sph<<<b, t, s>>>(g_idx_sph, p_idx_sph, g_str_sph, g_end_sph, dP1s, dP2s, dSP1s, dSP2s);
    b.x = bd; KERNEL_reorder_dem<<<b, t, s>>>(g_idx_dem, p_idx_dem, g_str_dem, g_end_dem, dP1d, dP2d, dSP1d, dSP2d);
    cudaDeviceSynchronize();
    cudaMemset(dP3s, 0, sizeof(part3) * num_part2_sph);
    cudaMemset(dP3d, 0, sizeof(part3) * num_part2_dem);
    cudaMemcpy(dP1s, dSP1s, sizeof(part1) * num_part2_sph, cudaMemcpyDeviceToDevice);
    cudaMemcpy(dP1d, dSP1d, sizeof(part1) * num_part2_dem, cudaMemcpyDeviceToDevice);
    b.x = bs; KERNEL_clc_mass_init_sph<<<b, t>>>(g_str_sph, g_end_sph, dSP1s, dSP2s, count);
    cudaDeviceSynchronize();
    if (kgc_solve > 0) gradient_correction_sph(g_str_sph, g_end_sph, dSP1s, dP3s);
    b.x = bs;
    KERNEL_clc_prep3D_coupling_sph<<<b, t>>>(g_str_sph, g_end_sph, dSP1s, dSP2s, g_str_dem, g_end_dem, dSP1d, dSP2d,
                                             count, time);
    b.x = bd;
    KERNEL_clc_prep3D_coupling_dem<<<b, t>>>(g_str_dem, g_end_dem, dSP1d, dSP2d, g_str_sph, g_end_sph, dSP1s, dSP2s,
                                             count, time);
    cudaDeviceSynchronize();
    b.x = bs; KERNEL_clc_prep3D_prep_sph<<<b, t>>>(g_str_sph, g_end_sph, dSP1s, dSP2s, dP3s, count);
    cudaDeviceSynchronize();
    b.x = bs; KERNEL_clc_prep3D_sph<<<b, t>>>(g_str_sph, g_end_sph, dSP1s, dSP2s, dP3s, count);
    cudaDeviceSynchronize();
    b.x = (num_part2 - 1) / t.x + 1;
    if ((noslip_bc == 1) || (penetration_solve == 1)) {
        KERNEL_boundary3D<<<b, t>>>(g_str, g_end, dSP1);
        cudaDeviceSynchronize();
    }
    b.x = bs; KERNEL_advection_force3D_sph<<<b, t>>>(1, g_str_sph, g_end_sph, dSP1s, dSP2s, dP3s);
    cudaDeviceSynchronize();
    b.x = bd; KERNEL_DEM_interaction3D_dem<<<b, t>>>(1, g_str_dem, g_end_dem, dSP1d, dP1d, dP3d, time);
    cudaDeviceSynchronize();
    b.x = bs;   // the reference sizes this launch by the SPH count
    KERNEL_DEM_coupling3D_dem<<<b, t>>>(1, g_str_dem, g_end_dem, dSP1d, dSP2d, dP3d, g_str_sph, g_end_sph, dSP1s,
                                        dSP2s, dP3s);
    cudaDeviceSynchronize();
    b.x = bs;
    KERNEL_SPH_coupling3D_sph<<<b, t>>>(1, g_str_sph, g_end_sph, dSP1s, dP3s, g_str_dem, g_end_dem, dSP1d, dP3d);
    cudaDeviceSynchronize();
    if (time_type == Pre_Cor) {
        b.x = bs; KERNEL_clc_projection_sph<<<b, t>>>(count, dt, time, dSP1s, dSP2s, dP3s);
        b.x = bd; KERNEL_clc_projection_dem<<<b, t>>>(count, dt, time, dSP1d, dSP2d, dP3d);
        cudaDeviceSynchronize();
    }
    if (count == 0) {
        b.x = bs; KERNEL_Neumann_boundary3D_sph<<<b, t>>>(g_str_sph, g_end_sph, dSP1s, dSP2s, dP3s);
        cudaDeviceSynchronize();
    }
    b.x = bs; KERNEL_PPE3D_sph<<<b, t>>>(dt, g_str_sph, g_end_sph, dSP1s, dSP2s, dP3s);
    cudaDeviceSynchronize();
    b.x = bs; KERNEL_PPE3D_calc_sph<<<b, t>>>(dt, g_str_sph, g_end_sph, dSP1s, dSP2s, dP3s);
    cudaDeviceSynchronize();
    b.x = bs; KERNEL_Neumann_boundary3D_sph<<<b, t>>>(g_str_sph, g_end_sph, dSP1s, dSP2s, dP3s);
    cudaDeviceSynchronize();
    b.x = bs; KERNEL_pressureforce3D_sph<<<b, t>>>(1, g_str_sph, g_end_sph, dSP1s, dSP2s, dP3s);
    cudaDeviceSynchronize();
    b.x = bs; KERNEL_time_update_projection_sph<<<b, t>>>(dt, dSP1s, dP1s, dSP2s, dP2s, dP3s);
    b.x = bd; KERNEL_time_update_projection_dem<<<b, t>>>(dt, dSP1d, dP1d, dSP2d, dP2d, dP3d);
    cudaDeviceSynchronize();
    if (open_boundary > 0) {
        b.x = bs;
        KERNEL_open_boundary_extrapolation3D_1_sph<<<b, t>>>(time, g_str_sph, g_end_sph, dP1s, dSP2s, dP3s, count, dt);
        cudaDeviceSynchronize();
        KERNEL_open_boundary_extrapolation3D_1_calc_sph<<<b, t>>>(time, g_str_sph, g_end_sph, dP1s, dSP2s, dP3s, count,
                                                                  dt);
        cudaDeviceSynchronize();
    }
    if (xsph_solve) {
        b.x = bs; KERNEL_xsph3D_sph<<<b, t>>>(1, g_str_sph, g_end_sph, dt, time, dP1s, dSP2s);
        cudaDeviceSynchronize();
        b.x = bs; KERNEL_xsph3D_calc_sph<<<b, t>>>(1, g_str_sph, g_end_sph, dt, time, dP1s, dSP2s);
        cudaDeviceSynchronize();
    }
}

// nsteps of isph_step_without_dem_walls (3-D ISPH-DEM input, decouple_stride 1)
extern "C" int ref_run_without_dem_walls(int nsteps) {
    if (loaded != 1) return -1;
    if (decouple_stride != 1 || dim != 3) return -2;
    cudaDeviceSynchronize();
    auto t0 = refh_now();
    for (int k = 0; k < nsteps; k++) {
        isph_step_without_dem_walls();
        time += dt;
        count++;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return -100;
    auto t1 = refh_now();
    last_ms = refh_ms(t0, t1);
    if (cudaGetLastError() != cudaSuccess) return -101;
    HCK(cudaMemcpy(fP1s, dP1s, num_part2_sph * sizeof(part1), cudaMemcpyDeviceToHost));
    HCK(cudaMemcpy(fP2s, dSP2s, num_part2_sph * sizeof(part2), cudaMemcpyDeviceToHost));
    HCK(cudaMemcpy(fP3s, dP3s, num_part2_sph * sizeof(part3), cudaMemcpyDeviceToHost));
    if (num_part2_dem) {
        HCK(cudaMemcpy(fP1d, dP1d, num_part2_dem * sizeof(part1), cudaMemcpyDeviceToHost));
        HCK(cudaMemcpy(fP2d, dSP2d, num_part2_dem * sizeof(part2), cudaMemcpyDeviceToHost));
        HCK(cudaMemcpy(fP3d, dP3d, num_part2_dem * sizeof(part3), cudaMemcpyDeviceToHost));
    }
    return 0;
}

extern "C" double ref_last_ms(void) { return last_ms; }

extern "C" int ref_counts(int* ns, int* nd, int* nijk) {
    *ns = num_part2_sph;
    *nd = num_part2_dem;
    nijk[0] = NI; nijk[1] = NJ; nijk[2] = NK;
    return 0;
}

// copy one field of the read-back state (which: 0 SPH, 1 DEM)
extern "C" int ref_get(int which, const char* name, double* out) {
    int n = which ? num_part2_dem : num_part2_sph;
    part1* P1 = which ? fP1d : fP1s;
    part2* P2 = which ? fP2d : fP2s;
    part3* P3 = which ? fP3d : fP3s;
    std::string f(name);
#define G1(nm, expr) if (f == nm) { for (int k = 0; k < n; k++) out[k] = (double)(expr); return 0; }
    G1("x", P1[k].x) G1("y", P1[k].y) G1("z", P1[k].z)
    G1("ux", P1[k].ux) G1("uy", P1[k].uy) G1("uz", P1[k].uz)
    G1("wx", P1[k].wx) G1("wy", P1[k].wy) G1("wz", P1[k].wz)
    G1("m", P1[k].m) G1("rho", P1[k].rho) G1("pres", P1[k].pres) G1("temp", P1[k].temp)
    G1("h", P1[k].h) G1("rad", P1[k].rad) G1("DEMpor", P1[k].DEMpor) G1("dDEMpor", P1[k].dDEMpor)
    G1("flt_s", P1[k].flt_s) G1("flt_sd", P1[k].flt_sd) G1("flt_sd2", P1[k].flt_sd_2)
    G1("pgfx", P1[k].pgf_x) G1("pgfy", P1[k].pgf_y) G1("pgfz", P1[k].pgf_z)
    G1("Fdx_df", P1[k].Fdx_df) G1("Fdy_df", P1[k].Fdy_df) G1("Fdz_df", P1[k].Fdz_df)
    G1("p_type", P1[k].p_type) G1("i_type", P1[k].i_type) G1("buffer_type", P1[k].buffer_type)
    G1("dem_idx", P1[k].dem_idx) G1("pid", P1[k].concn)
    G1("rho_ref", P2[k].rho_ref)
    G1("ftotalx", P3[k].ftotalx) G1("ftotaly", P3[k].ftotaly) G1("ftotalz", P3[k].ftotalz)
    G1("fpx", P3[k].fpx) G1("fpy", P3[k].fpy) G1("fpz", P3[k].fpz)
    G1("torqx", P3[k].torqx) G1("torqy", P3[k].torqy) G1("torqz", P3[k].torqz)
    G1("dtemp", P3[k].dtemp) G1("Q_sd", P1[k].Q_sd) G1("drho", P3[k].drho) G1("ftotal", P3[k].ftotal)
    G1("grad_rhox", P1[k].grad_rhox) G1("grad_rhoy", P1[k].grad_rhoy) G1("vis_t", P3[k].vis_t)
#undef G1
    if (f.rfind("ct_idx", 0) == 0) {   // ct_idx<s>
        int s = atoi(f.c_str() + 6);
        for (int k = 0; k < n; k++) out[k] = P1[k].ct_idx[s];
        return 0;
    }
    if (f.rfind("del_s", 0) == 0) {    // del_s<s>_<c>
        int s = atoi(f.c_str() + 5), c = atoi(strrchr(f.c_str(), '_') + 1);
        for (int k = 0; k < n; k++) out[k] = P1[k].del_s[s][c];
        return 0;
    }
    return -1;
}

// cell start/end and sorted cell index of the SPH set (last NNPS)
extern "C" int ref_get_cells(int which, int* gstr, int* gend, int* gidx) {
    int n = which ? num_part2_dem : num_part2_sph;
    if (cudaMemcpy(gstr, which ? g_str_dem : g_str_sph, sizeof(int) * num_cells, cudaMemcpyDeviceToHost) != cudaSuccess) return -100;
    if (cudaMemcpy(gend, which ? g_end_dem : g_end_sph, sizeof(int) * num_cells, cudaMemcpyDeviceToHost) != cudaSuccess) return -100;
    if (n && cudaMemcpy(gidx, which ? g_idx_dem : g_idx_sph, sizeof(int) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return -100;
    return num_cells;
}
