// io.cpp -- SOPHIA_gpu input/output formats on the host.
//
//   solv.txt  keyword scanner   function_init.cuh:216-615
//   input.txt column reader     function_init.cuh:704-891
//   data.txt  table reader      function_init.cuh:966-1182 (validated only)
//   DEM VTK   big-endian POLYDATA functions_OUTPUT.cuh:1135-1446
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "handle.h"

// Reference-compat preset: input/solv.txt of the reference plus every
// constant it hard-wires with #define (Parameters.cuh, functions_PROP.cuh,
// functions_NNPS.cuh:2-5, functions_DEM_BC.cuh, functions_BC.cuh:961-966).
void sphdem_io_params_default(SphdemParams* p) {
    std::memset(p, 0, sizeof(*p));
    p->solver_type = SPHDEM_ISPH;
    p->dim = 3;
    p->prop_table = 0;
    p->kernel_type = SPHDEM_KERNEL_WENDLAND6;
    p->flt_type = 0;
    p->rho_type = 1;            // Continuity
    p->time_type = 1;           // Predictor_Corrector
    p->fluid_type = 0;
    p->open_boundary = 1;
    p->simulation_type = 1;
    p->freq_cell = 1;
    p->flag_z_index = 0;
    p->flag_timestep_update = 0;
    p->nb_cell_type = 0;
    p->freq_filt = 40;
    p->freq_mass_sum = 1;
    p->freq_temp = 10;
    p->freq_output = 10000;
    p->fp_solve = 1;
    p->fv_solve = 1;
    p->fva_solve = 0;
    p->fg_solve = 1;
    p->fs_solve = 0;
    p->fb_solve = 0;
    p->con_solve = 0;
    p->boussinesq_solve = 0;
    p->interface_solve = 0;
    p->surf_model = 1;
    p->xsph_solve = 1;
    p->kgc_solve = 1;
    p->delSPH_solve = 2;
    p->delSPH_model = 0;
    p->pst_solve = 0;
    p->turbulence_model = 0;
    p->concn_solve = 0;
    p->min_iteration = 3;
    p->max_iteration = 10;
    p->penetration_solve = 0;
    p->switch_ptype = 0;
    p->noslip_bc = 0;
    p->decouple_stride = 1;
    p->ppe_mode = SPHDEM_PPE_REFERENCE;
    p->warm_start = SPHDEM_WARM_PREVIOUS;
    p->ppe_max_iter = 500;
    p->mlp_train_steps = 500;
    p->mlp_updates = 4;
    p->warm_hist = 8;
    p->mlp_seed = 0;
    p->mlp_lr = 3e-4;
    p->art_visc_alpha = 0.1;
    p->art_visc_beta = 0.02;
    p->delta_sph = 0.1;
    p->precision = SPHDEM_PREC_FP32;
    p->dem_wall_mask = 7;
    p->kappa = 2.0;
    p->p_ref = 0.0;
    p->gamma = 1.0;
    p->dt = 5.0e-7;
    p->time = 0.0;
    p->time_end = 5.0;
    for (int k = 0; k < 6; k++) p->margin[k] = 0.0;
    p->u_limit = 40.0;
    p->c_xsph = 0.1;
    p->c_repulsive = 0.00005;
    p->drho_th = 0.005;
    p->dp_th = 10.0;
    p->p_relaxation = 1.0;
    p->soundspeed = 200.0;
    p->rho0_eos = 1.784;
    p->ball_vel = 0.0;
    p->ppe_tol = 1e-6;
    p->rho_gas = 1.784;
    p->rho_liquid = 1000.0;
    p->mu_gas = 2.0e-5;
    p->mu_liquid = 1.0e-3;
    p->g_sph = 9.8;
    p->g_dem = 9.8;
    p->h_over_dx = 1.6;
    p->k_sph = 0.0518;
    p->cp_sph = 1006.4;
    p->k_dem = 2.5;
    p->cp_dem = 1068.0;
    p->dem_shear_modulus = 8.3e8;
    p->dem_poisson = 0.23;
    p->dem_damp_coef = 0.0535184;
    p->dem_friction_ratio = 0.5;
    p->dem_contact_range = 2.01;
    p->dem_search_range = 3.5;
    p->nu_gas = 2.0e-5 / 1.784;
    p->inlet_uz_mirror = 24.045;
    p->inlet_temp = 823.0;
    p->obc_L1 = -10.505;
    p->obc_L2 = -0.021;
    p->obc_L3 = 0.006;
    p->obc_L4 = 10.25;
    p->cyl_cx = 0.0;
    p->cyl_cy = 0.0;
    p->cyl_r = 0.0125;
    p->box_c[0] = 0.0;
    p->box_c[1] = 0.0;
    p->box_c[2] = -0.00176647182;
    p->box_L[0] = 1.15;
    p->box_L[1] = 1.015;
    p->box_L[2] = 0.03353294364;
    p->cone_c[0] = 0.0;
    p->cone_c[1] = 0.0;
    p->cone_c[2] = 0.0;
    p->cone_r1 = 0.0125;
    p->cone_r2 = 0.0018;
    p->cone_h = 0.01853294364;
    p->wall_rest_n = 0.9;
    p->wall_rest_s = -0.9;
    p->wall_mu_s = 0.10;
    p->wall_mu_rs = 0.2;
}

extern "C" int sphdem_params_default(SphdemParams* p) {
    if (!p) return SPHDEM_E_ARG;
    sphdem_io_params_default(p);
    return SPHDEM_OK;
}

// ---------------------------------------------------------------------------
// solv.txt: whitespace-token scanner.  Each recognised key consumes the
// same number of following tokens as the reference parser.
// ---------------------------------------------------------------------------
namespace {
struct Tok {
    std::vector<std::string> t;
    size_t k = 0;
    bool next(std::string& s) {
        if (k >= t.size()) return false;
        s = t[k++];
        return true;
    }
};
bool yesno(const std::string& s, int32_t* dst) {
    if (s == "YES") { *dst = 1; return true; }
    if (s == "NO") { *dst = 0; return true; }
    return false;
}
}  // namespace

extern "C" int sphdem_read_solv(const char* path, SphdemParams* p) {
    if (!path || !p) return SPHDEM_E_ARG;
    FILE* f = std::fopen(path, "r");
    if (!f) return SPHDEM_E_INPUT;
    Tok T;
    char buf[1024];
    while (std::fscanf(f, "%1023s", buf) == 1) T.t.emplace_back(buf);
    std::fclose(f);
    // read_solv_input starts by clearing these switches (function_init.cuh:218-237)
    p->solver_type = SPHDEM_WCSPH;
    p->fp_solve = p->fv_solve = p->fva_solve = p->fg_solve = p->fs_solve = p->fb_solve = 0;
    p->con_solve = p->boussinesq_solve = p->interface_solve = p->xsph_solve = p->kgc_solve = 0;
    p->delSPH_solve = p->pst_solve = p->turbulence_model = p->concn_solve = 0;
    p->c_xsph = 0.0;
    p->c_repulsive = 0.0;
    std::string s, v;
    auto skip = [&](int n) { for (int q = 0; q < n; q++) T.next(v); };
    while (T.next(s)) {
        if (s == "solver_type") {
            skip(2);
            if (v == "WCSPH") p->solver_type = SPHDEM_WCSPH;
            if (v == "ISPH") p->solver_type = SPHDEM_ISPH;
            if (v == "DFSPH") p->solver_type = SPHDEM_DFSPH;
        } else if (s == "dimension(1/2/3):") {
            skip(1); p->dim = std::atoi(v.c_str());
        } else if (s == "property_table(YES/NO):") {
            skip(1); yesno(v, &p->prop_table);
        } else if (s == "kernel") {
            skip(3);
            if (v == "Quartic") p->kernel_type = SPHDEM_KERNEL_QUARTIC;
            if (v == "Gaussian") p->kernel_type = SPHDEM_KERNEL_GAUSSIAN;
            if (v == "Quintic") p->kernel_type = SPHDEM_KERNEL_QUINTIC;
            if (v == "Wendland2") p->kernel_type = SPHDEM_KERNEL_WENDLAND2;
            if (v == "Wendland4") p->kernel_type = SPHDEM_KERNEL_WENDLAND4;
            if (v == "Wendland6") p->kernel_type = SPHDEM_KERNEL_WENDLAND6;
        } else if (s == "filter") {
            skip(3);
            if (v == "Shepard") p->flt_type = 0;
            if (v == "MLS") p->flt_type = 1;
        } else if (s == "density") {
            skip(3);
            if (v == "Direct") p->rho_type = 0;
            if (v == "Continuity") p->rho_type = 1;
        } else if (s == "time") {
            skip(3);
            if (v == "Euler") p->time_type = 0;
            if (v == "Predictor_Corrector") p->time_type = 1;
        } else if (s == "fluid") {
            skip(3);
            if (v == "Liquid") p->fluid_type = 0;
            if (v == "Gas") p->fluid_type = 1;
        } else if (s == "simulation") {
            skip(3);
            if (v == "Single_Phase") p->simulation_type = 1;
            if (v == "Two_Phase") p->simulation_type = 2;
        } else if (s == "open") {
            skip(3);
            if (v == "OPEN") p->open_boundary = 1;
            if (v == "PERIODIC") p->open_boundary = 2;
            if (v == "NO") p->open_boundary = 0;
        } else if (s == "pressure-force") {
            skip(2); yesno(v, &p->fp_solve);
        } else if (s == "viscous-force") {
            skip(2); yesno(v, &p->fv_solve);
        } else if (s == "turbulence-model") {
            skip(2);
            if (v == "Laminar") p->turbulence_model = 0;
            if (v == "k-lm") p->turbulence_model = 1;
            if (v == "k-e") p->turbulence_model = 2;
            if (v == "SPS") p->turbulence_model = 3;
            if (v == "HB") p->turbulence_model = 4;
        } else if (s == "artificial-viscous-force") {
            skip(2); yesno(v, &p->fva_solve);
        } else if (s == "gravitational-force") {
            skip(2); yesno(v, &p->fg_solve);
        } else if (s == "surface-tension-force") {
            skip(2); yesno(v, &p->fs_solve);
        } else if (s == "surface-tension-model") {
            skip(2);
            if (v == "Potential") p->surf_model = 1;
            if (v == "Curvature") p->surf_model = 2;
        } else if (s == "interface-sharpness-force") {
            skip(2); yesno(v, &p->interface_solve);
        } else if (s == "boundary-force") {
            skip(2); yesno(v, &p->fb_solve);
        } else if (s == "Conduction(YES/NO):") {
            skip(1); yesno(v, &p->con_solve);
        } else if (s == "Boussinesq-natural-convection") {
            skip(2); yesno(v, &p->boussinesq_solve);
        } else if (s == "Concentration-diffusion(YES/NO):") {
            skip(1); yesno(v, &p->concn_solve);
        } else if (s == "XSPH") {
            skip(2); yesno(v, &p->xsph_solve);
        } else if (s == "kernel-gradient-correction") {
            skip(2);
            if (v == "NO") p->kgc_solve = 0;
            if (v == "KGC") p->kgc_solve = 1;
            if (v == "FPM") p->kgc_solve = 2;
            if (v == "DFPM") p->kgc_solve = 3;
            if (v == "KGF") p->kgc_solve = 4;
        } else if (s == "delta-SPH") {
            skip(2);
            if (v == "NO") p->delSPH_solve = 0;
            if (v == "Molteni") p->delSPH_solve = 1;
            if (v == "Antuono") p->delSPH_solve = 2;
        } else if (s == "particle-shifting") {
            skip(2); yesno(v, &p->pst_solve);
        } else if (s == "penetration_box") {
            skip(2); yesno(v, &p->penetration_solve);
        } else if (s == "switch_ptype") {
            skip(2); yesno(v, &p->switch_ptype);
        } else if (s == "noslip_boundary") {
            skip(2); yesno(v, &p->noslip_bc);
        } else if (s == "reference-pressure") {
            skip(2); p->p_ref = std::atof(v.c_str());
        } else if (s == "sound-speed:") {
            skip(1); p->soundspeed = std::atof(v.c_str());
        } else if (s == "reference-density-eos:") {
            skip(1); p->rho0_eos = std::atof(v.c_str());
        } else if (s == "gamma") {
            skip(3); p->gamma = std::atof(v.c_str());
        } else if (s == "kappa:") {
            skip(1); p->kappa = std::atof(v.c_str());
        } else if (s == "XSPH-coefficient:") {
            skip(1); p->c_xsph = std::atof(v.c_str());
        } else if (s == "Boundary-coefficient:") {
            skip(1); p->c_repulsive = std::atof(v.c_str());
        } else if (s == "minimum-iteration:") {
            skip(1); p->min_iteration = std::atoi(v.c_str());
        } else if (s == "maximum-iteration:") {
            skip(1); p->max_iteration = std::atoi(v.c_str());
        } else if (s == "pressure-convergence") {
            skip(2); p->dp_th = std::atof(v.c_str());
        } else if (s == "density-convergence") {
            skip(2); p->drho_th = std::atof(v.c_str());
        } else if (s == "pressure-relaxation") {
            skip(2); p->p_relaxation = std::atof(v.c_str());
        } else if (s == "time-step") {
            skip(2); p->dt = std::atof(v.c_str());
        } else if (s == "start-time") {
            skip(2); p->time = std::atof(v.c_str());
        } else if (s == "end-time") {
            skip(2); p->time_end = std::atof(v.c_str());
        } else if (s == "ball-velocity") {
            skip(2); p->ball_vel = std::atof(v.c_str());
        } else if (s == "cell-initialization") {
            skip(2); p->freq_cell = std::atoi(v.c_str());
        } else if (s == "z-indexing") {
            skip(2); yesno(v, &p->flag_z_index);
        } else if (s == "timestep") {
            skip(2); yesno(v, &p->flag_timestep_update);
        } else if (s == "neighbor") {
            skip(3);
            if (v == "3X3") p->nb_cell_type = 0;
            if (v == "5X5") p->nb_cell_type = 1;
        } else if (s == "filtering") {
            skip(2); p->freq_filt = std::atoi(v.c_str());
        } else if (s == "density-renormalization") {
            skip(2); p->freq_mass_sum = std::atoi(v.c_str());
        } else if (s == "temperature-filtering") {
            skip(2); p->freq_temp = std::atoi(v.c_str());
        } else if (s == "plot-output") {
            skip(2); p->freq_output = std::atoi(v.c_str());
        } else if (s == "plot-variables:") {
            skip(1);
            int nplot = std::atoi(v.c_str());
            skip(nplot > 0 ? nplot : 0);
        } else if (s == "velocity-limit") {
            skip(2); p->u_limit = std::atof(v.c_str());
        } else if (s == "Xmargin(-):") {
            skip(1); p->margin[0] = std::atof(v.c_str());
        } else if (s == "Xmargin(+):") {
            skip(1); p->margin[1] = std::atof(v.c_str());
        } else if (s == "Ymargin(-):") {
            skip(1); p->margin[2] = std::atof(v.c_str());
        } else if (s == "Ymargin(+):") {
            skip(1); p->margin[3] = std::atof(v.c_str());
        } else if (s == "Zmargin(-):") {
            skip(1); p->margin[4] = std::atof(v.c_str());
        } else if (s == "Zmargin(+):") {
            skip(1); p->margin[5] = std::atof(v.c_str());
        } else if (s == "decouple-stride:") {
            skip(1); p->decouple_stride = std::atoi(v.c_str());
        }
    }
    return SPHDEM_OK;
}

// ---------------------------------------------------------------------------
// input.txt: first line = tab-separated integer column labels
// (function_init.cuh:704-739), then whitespace-separated values per row.
// Rows with p_type <= 1000 are SPH, the rest DEM (function_init.cuh:893-911).
// ---------------------------------------------------------------------------
int sphdem_io_read_input_txt(const char* path, SphdemHandle* h, const SphdemParams* p) {
    (void)p;
    FILE* f = std::fopen(path, "r");
    if (!f) return SPHDEM_E_INPUT;
    char line[4096];
    if (!std::fgets(line, sizeof(line), f)) { std::fclose(f); return SPHDEM_E_INPUT; }
    std::vector<int> lbl;
    for (char* tok = std::strtok(line, "\t"); tok; tok = std::strtok(nullptr, "\t")) {
        int v = std::atoi(tok);
        lbl.push_back(v);
    }
    int nov = (int)lbl.size();
    if (nov == 0) { std::fclose(f); return SPHDEM_E_INPUT; }
    for (int v : lbl)
        if (v < 1 || v > 36) { std::fclose(f); return SPHDEM_E_INPUT; }
    std::vector<std::vector<double>> col(37);
    char tokbuf[256];
    int nrow = 0;
    bool done = false;
    while (!done) {
        std::vector<double> row(nov);
        for (int j = 0; j < nov; j++) {
            if (std::fscanf(f, "%255s", tokbuf) != 1) {
                if (j != 0) { std::fclose(f); return SPHDEM_E_INPUT; }  // truncated row
                done = true;
                break;
            }
            char* endp = nullptr;
            double val = std::strtod(tokbuf, &endp);
            if (endp == tokbuf) { std::fclose(f); return SPHDEM_E_INPUT; }
            row[j] = val;
        }
        if (done) break;
        for (int j = 0; j < nov; j++) col[lbl[j]].push_back(row[j]);
        nrow++;
    }
    std::fclose(f);
    if (nrow == 0) return SPHDEM_E_INPUT;
    auto get = [&](int c, int r, double dflt) { return col[c].empty() ? dflt : col[c][r]; };
    // split by p_type (label 8)
    std::vector<int> isdem(nrow);
    int ns = 0, nd = 0;
    for (int r = 0; r < nrow; r++) {
        int pt = (int)get(8, r, 0);
        isdem[r] = pt > 1000;
        if (isdem[r]) nd++; else ns++;
    }
    h->ns = ns;
    h->nd = nd;
    struct Map { int lbl; int field; };
    const Map real_map[] = {{1, SPHDEM_F_X}, {2, SPHDEM_F_Y}, {3, SPHDEM_F_Z}, {4, SPHDEM_F_UX}, {5, SPHDEM_F_UY},
                            {6, SPHDEM_F_UZ}, {7, SPHDEM_F_M}, {9, SPHDEM_F_H}, {10, SPHDEM_F_TEMP},
                            {11, SPHDEM_F_PRES}, {12, SPHDEM_F_RHO}, {26, SPHDEM_F_FLT_S}, {27, SPHDEM_F_RAD},
                            {28, SPHDEM_F_RI}, {30, SPHDEM_F_WX}, {31, SPHDEM_F_WY}, {32, SPHDEM_F_WZ},
                            {33, SPHDEM_F_TEMP1}, {34, SPHDEM_F_TEMP2}, {35, SPHDEM_F_TEMP3}};
    for (const Map& m : real_map) {
        std::vector<double> a[2];
        for (int r = 0; r < nrow; r++) a[isdem[r]].push_back(get(m.lbl, r, 0.0));
        h->stage_d[0][m.field] = a[0];
        h->stage_d[1][m.field] = a[1];
    }
    const Map int_map[] = {{8, SPHDEM_F_PTYPE}, {29, SPHDEM_F_DEM_IDX}};
    for (const Map& m : int_map) {
        std::vector<int> a[2];
        for (int r = 0; r < nrow; r++) a[isdem[r]].push_back((int)get(m.lbl, r, 0.0));
        h->stage_i[0][m.field] = a[0];
        h->stage_i[1][m.field] = a[1];
    }
    h->file_x = col[1].empty() ? std::vector<double>(nrow, 0.0) : col[1];
    h->file_y = col[2].empty() ? std::vector<double>(nrow, 0.0) : col[2];
    h->file_z = col[3].empty() ? std::vector<double>(nrow, 0.0) : col[3];
    h->file_h0 = get(9, 0, 0.0);
    h->have_file_order = true;
    return SPHDEM_OK;
}

// data.txt: "#p_type N" blocks with //T, //h, //k, //mu comma lists,
// closed by "#end" (function_init.cuh:966-1182).  Only the format is
// checked: property tables are not used by the supported switch sets.
int sphdem_io_check_table(const char* path) {
    FILE* f = std::fopen(path, "r");
    if (!f) return SPHDEM_OK;  // the reference reads it unconditionally; absence is tolerated here
    char line[1024];
    int open = 0;
    while (std::fgets(line, sizeof(line), f)) {
        if (!std::strncmp(line, "#p_type", 7)) {
            if (open) { std::fclose(f); return SPHDEM_E_INPUT; }
            open = 1;
        } else if (!std::strncmp(line, "#end", 4)) {
            if (!open) { std::fclose(f); return SPHDEM_E_INPUT; }
            open = 0;
        }
    }
    std::fclose(f);
    return open ? SPHDEM_E_INPUT : SPHDEM_OK;
}

// ---------------------------------------------------------------------------
// DEM VTK (save_plot_fluid_vtk_bin_solid_dem)
// ---------------------------------------------------------------------------
static float be_float(double v) {
    float f = (float)v;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u = (u >> 24) | ((u >> 8) & 0xff00u) | ((u << 8) & 0xff0000u) | (u << 24);
    std::memcpy(&f, &u, 4);
    return f;
}

int sphdem_io_write_vtk_dem(const char* path, int n, const double* x, const double* y, const double* z,
                            const int* itype, const int* ptype, const int* dem_idx, const double* magf,
                            const double* eliz, const double* por, const double* uz, const double* qsd,
                            const double* ftz, const double* temp, const double* rad, const double* dtemp) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return SPHDEM_E_INPUT;
    int np = 0;
    for (int i = 0; i < n; i++)
        if (dem_idx[i] > 0) np++;
    std::fprintf(f, "# vtk DataFile Version 3.0\n");
    std::fprintf(f, "Print out results in vtk format\n");
    std::fprintf(f, "BINARY\n");
    std::fprintf(f, "DATASET POLYDATA\n");
    std::fprintf(f, "POINTS\t%d\tfloat\n", np);
    for (int i = 0; i < n; i++) {
        if (ptype[i] <= 1000) continue;
        float v[3] = {be_float(x[i]), be_float(y[i]), be_float(z[i])};
        std::fwrite(v, sizeof(float), 3, f);
    }
    std::fprintf(f, "POINT_DATA\t%d\n", np);
    std::fprintf(f, "FIELD FieldData\t10\n");
    auto arr = [&](const char* name, const double* a, const int* ai) {
        std::fprintf(f, "%s\t1\t%d\tfloat\n", name, np);
        for (int i = 0; i < n; i++) {
            if (ptype[i] <= 1000) continue;
            float v = be_float(a ? a[i] : (double)ai[i]);
            std::fwrite(&v, sizeof(float), 1, f);
        }
    };
    arr("itype", nullptr, itype);
    arr("mag_uijf", magf, nullptr);
    arr("Euler", eliz, nullptr);
    arr("porosity", por, nullptr);
    arr("uz", uz, nullptr);
    arr("Q_sd", qsd, nullptr);
    arr("ftotal_z", ftz, nullptr);
    arr("temperature_surface", temp, nullptr);
    arr("rad", rad, nullptr);
    arr("dtemp_dt", dtemp, nullptr);
    std::fclose(f);
    return SPHDEM_OK;
}

static int be_int(int v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u = (u >> 24) | ((u >> 8) & 0xff00u) | ((u << 8) & 0xff0000u) | (u << 24);
    std::memcpy(&v, &u, 4);
    return v;
}

// The reference's fluid writer (functions_OUTPUT.cuh:445-651): fluid
// particles only (p_type 1), big-endian float positions, then nine point
// arrays.  Its conv_rate and cond_rate arrays print part1::Q_sdf and
// part1::Q_f, which no kernel of the compiled tree assigns, so they are
// zero there and zero here.
int sphdem_io_write_vtk_fluid(const char* path, int n, const int* ptype, const double* x, const double* y,
                              const double* z, const double* por, const double* pres, const double* dtemp,
                              const int* btype, const double* rho, const double* temp, const double* uz) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return SPHDEM_E_INPUT;
    int np = 0;
    for (int i = 0; i < n; i++)
        if (ptype[i] == 1) np++;
    std::fprintf(f, "# vtk DataFile Version 3.0\n");
    std::fprintf(f, "Print out results in vtk format\n");
    std::fprintf(f, "BINARY\n");
    std::fprintf(f, "DATASET POLYDATA\n");
    std::fprintf(f, "POINTS\t%d\tfloat\n", np);
    for (int i = 0; i < n; i++) {
        if (ptype[i] != 1) continue;
        float v[3] = {be_float(x[i]), be_float(y[i]), be_float(z[i])};
        std::fwrite(v, sizeof(float), 3, f);
    }
    std::fprintf(f, "POINT_DATA\t%d\n", np);
    std::fprintf(f, "FIELD FieldData\t9\n");
    auto arr = [&](const char* name, const double* a) {
        std::fprintf(f, "%s\t1\t%d\tfloat\n", name, np);
        for (int i = 0; i < n; i++) {
            if (ptype[i] != 1) continue;
            float v = be_float(a ? a[i] : 0.0);
            std::fwrite(&v, sizeof(float), 1, f);
        }
    };
    arr("porosity", por);
    arr("conv_rate", nullptr);
    arr("pressure", pres);
    arr("cond_rate", nullptr);
    arr("dtemp", dtemp);
    std::fprintf(f, "buffer_type\t1\t%d\tint\n", np);
    for (int i = 0; i < n; i++) {
        if (ptype[i] != 1) continue;
        int v = be_int(btype[i]);
        std::fwrite(&v, sizeof(int), 1, f);
    }
    arr("density", rho);
    arr("temperature", temp);
    arr("uz", uz);
    std::fclose(f);
    return SPHDEM_OK;
}

// ---------------------------------------------------------------------------
// host-only input.txt access
// ---------------------------------------------------------------------------
extern "C" int sphdem_input_counts(const char* path, int32_t* ns, int32_t* nd) {
    if (!path || !ns || !nd) return SPHDEM_E_ARG;
    SphdemHandle h;
    int r = sphdem_io_read_input_txt(path, &h, nullptr);
    if (r) return r;
    *ns = h.ns;
    *nd = h.nd;
    return SPHDEM_OK;
}

extern "C" int sphdem_input_column(const char* path, int which, int field, void* dst, size_t bytes) {
    if (!path || !dst || (which != 0 && which != 1)) return SPHDEM_E_ARG;
    SphdemHandle h;
    int r = sphdem_io_read_input_txt(path, &h, nullptr);
    if (r) return r;
    int n = which ? h.nd : h.ns;
    auto itd = h.stage_d[which].find(field);
    if (itd != h.stage_d[which].end()) {
        if (bytes != sizeof(double) * (size_t)n) return SPHDEM_E_ARG;
        std::memcpy(dst, itd->second.data(), bytes);
        return SPHDEM_OK;
    }
    auto iti = h.stage_i[which].find(field);
    if (iti != h.stage_i[which].end()) {
        if (bytes != sizeof(int) * (size_t)n) return SPHDEM_E_ARG;
        std::memcpy(dst, iti->second.data(), bytes);
        return SPHDEM_OK;
    }
    return SPHDEM_E_ARG;
}
