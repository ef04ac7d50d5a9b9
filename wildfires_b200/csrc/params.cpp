// params.cpp -- parameter files, derived grid arrays, terrain / immersed-
// boundary tables and the raw binary field files, on the host.
//
// The `key = value` format is the reference's (src/cu/parameters.cu:13-415):
// the record is zeroed, defaults are set (:39-76), then every line is tested
// against every key with strncmp over the reference's prefix length and read
// with sscanf at the reference's value offset, so later lines override earlier
// ones and unknown keys are ignored.  Derived arrays follow :416-523, the
// terrain and immersed-boundary tables ibm.cu:3-95, the z grids
// functions.cu:58-80, the wavenumbers utils.cu:32-51.  Field files follow
// input.cu:3-58 and output.cu:3-44.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "wf_internal.h"

namespace {

enum Kind { KI, KD, KS32, KS64 };

struct Key {
    const char *prefix;  // text the line must start with (first `n` characters)
    int n;               // compared length
    int off;             // offset of the value in the line
    Kind kind;
    size_t member;       // offsetof(Parameters, member)
};

#define M(f) offsetof(Parameters, f)
// Prefix lengths and value offsets are those of the reference parser.
const Key kKeys[] = {
    {"Nx =", 4, 5, KI, M(Nx)}, {"Ny =", 4, 5, KI, M(Ny)}, {"Nz =", 4, 5, KI, M(Nz)},
    {"Nt =", 4, 5, KI, M(Nt)}, {"NT =", 4, 5, KI, M(NT)},
    {"x_min =", 7, 8, KD, M(x_min)}, {"x_max =", 7, 8, KD, M(x_max)},
    {"y_min =", 7, 8, KD, M(y_min)}, {"y_max =", 7, 8, KD, M(y_max)},
    {"z_min =", 7, 8, KD, M(z_min)}, {"z_max =", 7, 8, KD, M(z_max)},
    {"t_min =", 7, 8, KD, M(t_min)}, {"t_max =", 7, 8, KD, M(t_max)},
    {"nu =", 4, 5, KD, M(nu)}, {"mu =", 4, 5, KD, M(mu)}, {"u_r =", 5, 6, KD, M(u_r)},
    {"z_r =", 5, 6, KD, M(z_r)}, {"alpha_u =", 9, 10, KD, M(alpha_u)}, {"alpha =", 7, 8, KD, M(alpha)},
    {"T_inf =", 7, 8, KD, M(T_inf)}, {"T_0 =", 5, 6, KD, M(T_0)}, {"T_source =", 10, 11, KD, M(T_source)},
    {"T0_shape =", 10, 11, KS32, M(T0_shape)},
    {"T0_x_start =", 12, 13, KD, M(T0_x_start)}, {"T0_x_end =", 10, 11, KD, M(T0_x_end)},
    {"T0_y_start =", 12, 13, KD, M(T0_y_start)}, {"T0_y_end =", 10, 11, KD, M(T0_y_end)},
    {"T0_z_start =", 12, 13, KD, M(T0_z_start)}, {"T0_z_end =", 10, 11, KD, M(T0_z_end)},
    {"Y0_x_start =", 12, 13, KD, M(Y0_x_start)}, {"Y0_x_end =", 10, 11, KD, M(Y0_x_end)},
    {"Y0_y_start =", 12, 13, KD, M(Y0_y_start)}, {"Y0_y_end =", 10, 11, KD, M(Y0_y_end)},
    {"Y0_xa =", 7, 8, KD, M(Y0_xa)}, {"Y0_ya =", 7, 8, KD, M(Y0_ya)},
    {"Y_h =", 5, 6, KD, M(Y_h)}, {"Y_f =", 5, 6, KD, M(Y_f)}, {"C_d =", 5, 6, KD, M(C_d)},
    {"alpha_s =", 9, 10, KD, M(alpha_s)}, {"sigma_s =", 9, 10, KD, M(sigma_s)},
    {"H_C =", 5, 6, KD, M(H_C)}, {"A =", 3, 4, KD, M(A)}, {"T_act =", 7, 8, KD, M(T_act)},
    {"T_pc =", 6, 7, KD, M(T_pc)}, {"h_c =", 5, 6, KD, M(h_c)}, {"c_p =", 5, 6, KD, M(c_p)},
    {"rho_inf =", 9, 10, KD, M(rho_inf)}, {"U0_type =", 9, 10, KS32, M(U0_type)},
    {"T0_shape =", 10, 11, KS32, M(T0_shape)}, {"g =", 3, 4, KD, M(g)}, {"C_s =", 5, 6, KD, M(C_s)},
    {"Pr =", 4, 5, KD, M(Pr)}, {"p_top =", 7, 8, KD, M(p_top)}, {"method =", 8, 9, KS32, M(method)},
    {"threads =", 9, 10, KI, M(n_threads)},
    {"T_min =", 6, 7, KD, M(T_min)}, {"T_max =", 6, 7, KD, M(T_max)},
    {"Y_min =", 6, 7, KD, M(Y_min)}, {"Y_max =", 6, 7, KD, M(Y_max)},
    {"topo_shape =", 11, 12, KS32, M(topo_shape)},
    {"u_dead_nodes =", 13, 14, KD, M(u_dead_nodes)}, {"v_dead_nodes =", 13, 14, KD, M(v_dead_nodes)},
    {"w_dead_nodes =", 13, 14, KD, M(w_dead_nodes)}, {"T_dead_nodes =", 13, 14, KD, M(T_dead_nodes)},
    {"Y_dead_nodes =", 13, 14, KD, M(Y_dead_nodes)},
    {"hill_center_x =", 14, 15, KD, M(hill_center_x)}, {"hill_center_y =", 14, 15, KD, M(hill_center_y)},
    {"hill_length =", 12, 13, KD, M(hill_length)}, {"hill_width =", 11, 12, KD, M(hill_width)},
    {"hill_height =", 12, 13, KD, M(hill_height)},
    {"t_source_start =", 16, 17, KD, M(t_source_start)}, {"t_source_end =", 14, 15, KD, M(t_source_end)},
    {"T_source_shape =", 16, 17, KS32, M(T_source_shape)}, {"delta =", 7, 8, KD, M(delta)},
    {"k =", 3, 4, KD, M(k)}, {"variable_density =", 17, 18, KI, M(variable_density)},
    {"pressure_solver_tol =", 21, 22, KD, M(pressure_solver_tol)},
    {"pressure_solver_iter =", 22, 23, KI, M(pressure_solver_iter)},
    {"pressure_solver_log =", 21, 22, KI, M(pressure_solver_log)},
    {"z_domain =", 10, 11, KI, M(z_domain)}, {"k_nu_grid =", 11, 12, KD, M(k_nu_grid)},
    {"k_transition =", 14, 15, KI, M(k_transition)}, {"z_transition =", 14, 15, KD, M(z_transition)},
    {"input_path =", 12, 13, KS64, M(input_path)},
    {"velocity_correction_fd =", 24, 25, KI, M(velocity_correction_fd)},
    {"time_step_log =", 15, 16, KI, M(time_step_log)},
    {"temperature_convection =", 24, 25, KI, M(temperature_convection)},
    {"TS_x_start =", 12, 13, KD, M(TS_x_start)}, {"TS_x_end =", 10, 11, KD, M(TS_x_end)},
    {"TS_y_start =", 12, 13, KD, M(TS_y_start)}, {"TS_y_end =", 10, 11, KD, M(TS_y_end)},
    {"TS_z_start =", 12, 13, KD, M(TS_z_start)}, {"TS_z_end =", 10, 11, KD, M(TS_z_end)},
    {"sutherland_viscosity =", 22, 23, KI, M(sutherland_viscosity)},
    {"sutherland_conductivity =", 25, 26, KI, M(sutherland_conductivity)},
};
#undef M

const double kPi = 3.14159265358979323846;

void set_defaults(Parameters *P)
{
    P->mu = 1.802e-5;
    P->nu = 1.47e-5;
    P->z_r = 2.0;
    P->alpha_u = 1.0 / 7.0;
    P->alpha = 2.009e-5;
    P->T_inf = 288.15;
    P->C_d = 0.15;
    P->H_C = 21e6;
    P->A = 1e9;
    P->T_act = 18040.8533;
    P->T_pc = 523.0;
    P->T_0 = 1000.0;
    P->h_c = 1.42;
    P->c_p = 1007.0;
    P->k = 0.02476;
    P->delta = 0.1;
    P->rho_inf = 1.225;
    P->g = -9.807;
    P->C_s = 0.2;
    P->Pr = 0.7329;
    P->variable_density = 1;
    P->pressure_solver_tol = 1e-10;
    P->pressure_solver_iter = 50;
    P->pressure_solver_log = 0;
    P->n_threads = 1;
    P->T_min = 288.15;
    P->T_max = 2500.0;
    P->Y_min = 0.0;
    P->Y_max = 1.0;
    P->u_dead_nodes = 0.0;
    P->v_dead_nodes = 0.0;
    P->w_dead_nodes = 0.0;
    P->T_dead_nodes = 288.15;
    P->Y_dead_nodes = 0.0;
    P->input_path[0] = '\0';
    P->velocity_correction_fd = 0;
    P->time_step_log = 100;
    P->temperature_convection = 1;
}

void parse_line(Parameters *P, const char *line)
{
    char *base = reinterpret_cast<char *>(P);
    for (const Key &k : kKeys) {
        if (strncmp(line, k.prefix, k.n) != 0) continue;
        const char *v = line + k.off;
        if ((size_t)k.off > strlen(line)) continue;
        switch (k.kind) {
        case KI: sscanf(v, "%d", reinterpret_cast<int *>(base + k.member)); break;
        case KD: sscanf(v, "%lf", reinterpret_cast<double *>(base + k.member)); break;
        case KS32: sscanf(v, "%31s", base + k.member); break;
        case KS64: sscanf(v, "%63s", base + k.member); break;
        }
    }
}

void fft_freq(double *f, int n, double d)
{
    if (n % 2 == 0) {
        const int h = n / 2;
        for (int i = 0; i < h; i++) f[i] = i / (n * d);
        for (int i = h; i < n; i++) f[i] = (i - n) / (n * d);
    } else {
        const int h = (n - 1) / 2;
        for (int i = 0; i <= h; i++) f[i] = i / (n * d);
        for (int i = h + 1; i < n; i++) f[i] = (i - n) / (n * d);
    }
}

// cut nodes, height above terrain, fuel storage height (ibm.cu:57-95)
void immersed_boundary(Parameters *P)
{
    const int Nx = P->Nx, Ny = P->Ny, Nz = P->Nz;
    int nzy_max = 0;
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++) {
            const size_t c = (size_t)j + (size_t)Ny * i;
            const double topo = P->topography[c];
            P->cut_nodes[c] = 0;
            P->Nz_Y[c] = 0;
            for (int k = 0; k < Nz; k++) {
                const double dz = (k < Nz - 1) ? P->z[k + 1] - P->z[k] : P->z[k] - P->z[k - 1];
                if ((topo - dz) <= P->z[k] && P->z[k] <= topo) P->cut_nodes[c] = k;
                const double d = P->z[k] - topo;
                P->z_ibm[(size_t)k + (size_t)Nz * c] = d > 0.0 ? d : 0.0;
                if (P->z[k] <= topo + P->Y_h) P->Nz_Y[c] = k + 1;
            }
            if (P->Nz_Y[c] > nzy_max) nzy_max = P->Nz_Y[c];
        }
    P->Nz_Y_max = nzy_max;
}

template <class T> T *alloc_n(size_t n) { return static_cast<T *>(calloc(n ? n : 1, sizeof(T))); }

wf_status fill_derived(Parameters *P)
{
    const int Nx = P->Nx, Ny = P->Ny, Nz = P->Nz, Nt = P->Nt;
    if (Nx < 4 || Ny < 4 || Nz < 4 || Nt < 1) {
        wf::set_error("parameters: need Nx, Ny, Nz >= 4 and Nt >= 1 (got %d, %d, %d, %d)", Nx, Ny, Nz, Nt);
        return WF_ERR_PARSE;
    }
    if (P->NT < 1) P->NT = Nt;   // the reference divides by NT (solver.cu:245)
    P->x = alloc_n<double>(Nx);
    P->y = alloc_n<double>(Ny);
    P->z = alloc_n<double>(Nz);
    P->t = alloc_n<double>((size_t)Nt + 1);
    P->r = alloc_n<double>(Nx - 1);
    P->s = alloc_n<double>(Ny - 1);
    P->kx = alloc_n<double>(Nx - 1);
    P->ky = alloc_n<double>(Ny - 1);
    P->cut_nodes = alloc_n<int>((size_t)Nx * Ny);
    P->z_ibm = alloc_n<double>((size_t)Nx * Ny * Nz);
    P->topography = alloc_n<double>((size_t)Nx * Ny);
    P->Nz_Y = alloc_n<int>((size_t)Nx * Ny);
    if (!P->x || !P->y || !P->z || !P->t || !P->r || !P->s || !P->kx || !P->ky || !P->cut_nodes || !P->z_ibm ||
        !P->topography || !P->Nz_Y) {
        wf::set_error("parameters: host allocation failed");
        return WF_ERR_OOM;
    }
    P->dx = (P->x_max - P->x_min) / (Nx - 1);
    P->dy = (P->y_max - P->y_min) / (Ny - 1);
    P->dz = (P->z_max - P->z_min) / (Nz - 1);
    P->dt = (P->t_max - P->t_min) / Nt;
    fft_freq(P->r, Nx - 1, 1.0 / (Nx - 1));
    fft_freq(P->s, Ny - 1, 1.0 / (Ny - 1));
    for (int n = 0; n <= Nt; n++) P->t[n] = P->t_min + n * P->dt;
    for (int i = 0; i < Nx; i++) {
        P->x[i] = P->x_min + i * P->dx;
        if (i < Nx - 1) P->kx[i] = 2 * kPi * P->r[i] / (P->x_max - P->x_min);
    }
    for (int j = 0; j < Ny; j++) {
        P->y[j] = P->y_min + j * P->dy;
        if (j < Ny - 1) P->ky[j] = 2 * kPi * P->s[j] / (P->y_max - P->y_min);
    }
    if (P->z_domain == 0) {
        for (int k = 0; k < Nz; k++) P->z[k] = P->z_min + k * P->dz;
    } else if (P->z_domain == 1) {
        const double dz = (P->z_max - P->z_min) / (Nz - 1);
        for (int k = 0; k < Nz; k++)
            P->z[k] = (P->z_max - P->z_min) * (exp(P->k_nu_grid * k * dz / (P->z_max - P->z_min)) - 1) /
                          (exp(P->k_nu_grid) - 1) + P->z_min;
    } else if (P->z_domain == 2) {
        const double dz1 = (P->z_transition - P->z_min) / (P->k_transition - 1);
        const double dz2 = (P->z_max - P->z_transition) / (Nz - P->k_transition - 1);
        for (int k = 0; k < Nz; k++)
            P->z[k] = (k <= P->k_transition) ? P->z_min + k * dz1 : P->z_transition + (k - P->k_transition) * dz2;
    }
    P->T0_x_center = (P->T0_x_start + P->T0_x_end) / 2;
    P->T0_y_center = (P->T0_y_start + P->T0_y_end) / 2;
    P->T0_z_center = 0.0;
    P->T0_length = P->T0_x_end - P->T0_x_start;
    P->T0_width = P->T0_y_end - P->T0_y_start;
    P->T0_height = P->T0_z_end - P->T0_z_start;
    P->TS_x_center = (P->TS_x_start + P->TS_x_end) / 2.0;
    P->TS_y_center = (P->TS_y_start + P->TS_y_end) / 2.0;
    P->TS_z_center = 0.0;
    P->TS_length = P->TS_x_end - P->TS_x_start;
    P->TS_width = P->TS_y_end - P->TS_y_start;
    P->TS_height = P->TS_z_end - P->TS_z_start;
    const bool hill = strcmp(P->topo_shape, "hill") == 0;
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++) {
            double h = 0.0;
            if (hill)   // simple_hill with the reference's gaussian (functions.cu:22-24)
                h = P->hill_height * exp(-pow((P->x[i] - P->hill_center_x) / P->hill_length, 2.0) -
                                         pow((P->y[j] - P->hill_center_y) / P->hill_width, 2.0) -
                                         pow((0.0 - 0.0) / 1.0, 2.0));
            P->topography[(size_t)j + (size_t)Ny * i] = h;
        }
    immersed_boundary(P);
    const int size = Nx * Ny * Nz;
    P->field_indexes.u = 0;
    P->field_indexes.v = size;
    P->field_indexes.w = 2 * size;
    P->field_indexes.T = 3 * size;
    P->field_indexes.Y = 4 * size;
    int *ti = &P->turbulence_indexes.rho;
    for (int q = 0; q < 19; q++) ti[q] = q * size;
    return WF_OK;
}

wf_status read_raw(const char *path, double *dst, size_t n)
{
    FILE *f = fopen(path, "rb");
    if (!f) {
        wf::set_error("cannot open %s", path);
        return WF_ERR_IO;
    }
    const size_t r = fread(dst, sizeof(double), n, f);
    fclose(f);
    if (r != n) {
        wf::set_error("%s: expected %zu values, read %zu", path, n, r);
        return WF_ERR_IO;
    }
    return WF_OK;
}

wf_status write_raw(const char *path, const double *src, size_t n)
{
    FILE *f = fopen(path, "wb");
    if (!f) {
        wf::set_error("cannot create %s", path);
        return WF_ERR_IO;
    }
    const size_t w = fwrite(src, sizeof(double), n, f);
    fclose(f);
    if (w != n) {
        wf::set_error("%s: short write", path);
        return WF_ERR_IO;
    }
    return WF_OK;
}

}  // namespace

extern "C" {

wf_status wf_read_parameters(const char *path, Parameters *P)
{
    if (!path || !P) {
        wf::set_error("wf_read_parameters: null argument");
        return WF_ERR_ARG;
    }
    FILE *f = fopen(path, "r");
    if (!f) {
        wf::set_error("cannot open parameter file %s", path);
        return WF_ERR_IO;
    }
    memset(P, 0, sizeof(*P));
    set_defaults(P);
    char line[512];
    while (fgets(line, sizeof(line), f)) parse_line(P, line);
    fclose(f);
    const wf_status st = fill_derived(P);
    if (st != WF_OK) wf_free_parameters(P);
    return st;
}

void wf_free_parameters(Parameters *P)
{
    if (!P) return;
    free(P->x); free(P->y); free(P->z); free(P->t); free(P->r); free(P->s);
    free(P->kx); free(P->ky); free(P->cut_nodes); free(P->z_ibm); free(P->topography); free(P->Nz_Y);
    P->x = P->y = P->z = P->t = P->r = P->s = P->kx = P->ky = P->z_ibm = P->topography = nullptr;
    P->cut_nodes = P->Nz_Y = nullptr;
}

wf_status wf_set_topography(Parameters *P, const double *topo)
{
    if (!P || !topo || !P->topography || !P->z_ibm) {
        wf::set_error("wf_set_topography: invalid argument");
        return WF_ERR_ARG;
    }
    memcpy(P->topography, topo, sizeof(double) * (size_t)P->Nx * P->Ny);
    immersed_boundary(P);
    return WF_OK;
}

size_t wf_state_size(const Parameters *P)
{
    if (!P) return 0;
    return (size_t)4 * P->Nx * P->Ny * P->Nz + (size_t)P->Nx * P->Ny * P->Nz_Y_max;
}

wf_status wf_load_fields(const Parameters *P, const char *dir, double *y, double *pr)
{
    if (!P || !dir || !y || !pr) {
        wf::set_error("wf_load_fields: null argument");
        return WF_ERR_ARG;
    }
    const size_t N = (size_t)P->Nx * P->Ny * P->Nz, NY = (size_t)P->Nx * P->Ny * P->Nz_Y_max;
    const char *names[6] = {"u", "v", "w", "T", "Y", "p"};
    for (int q = 0; q < 6; q++) {
        char path[1024];
        snprintf(path, sizeof(path), "%s%s.bin", dir, names[q]);
        double *dst = (q < 5) ? y + q * N : pr;
        const size_t n = (q == 4) ? NY : N;
        const wf_status st = read_raw(path, dst, n);
        if (st) return st;
    }
    return WF_OK;
}

wf_status wf_save_domain(const Parameters *P, const char *dir)
{
    if (!P || !dir || !P->x || !P->y || !P->z) {
        wf::set_error("wf_save_domain: null argument or record without grid arrays");
        return WF_ERR_ARG;
    }
    const int NT = P->NT > 0 ? P->NT : P->Nt;
    std::vector<double> ts;
    for (int n = 0; n <= P->Nt; n++)
        if (n % NT == 0 || n == P->Nt) ts.push_back(P->t ? P->t[n] : P->t_min + n * P->dt);
    const double *src[4] = {P->x, P->y, P->z, ts.data()};
    const size_t cnt[4] = {(size_t)P->Nx, (size_t)P->Ny, (size_t)P->Nz, ts.size()};
    const char *names[4] = {"x", "y", "z", "t"};
    for (int q = 0; q < 4; q++) {
        char path[1024];
        snprintf(path, sizeof(path), "%s%s.bin", dir, names[q]);
        const wf_status st = write_raw(path, src[q], cnt[q]);
        if (st) return st;
    }
    return WF_OK;
}

wf_status wf_save_topography(const Parameters *P, const char *dir)
{
    if (!P || !dir || !P->topography || !P->Nz_Y) {
        wf::set_error("wf_save_topography: null argument or record without terrain arrays");
        return WF_ERR_ARG;
    }
    const size_t n = (size_t)P->Nx * P->Ny;
    char path[1024];
    snprintf(path, sizeof(path), "%stopography.bin", dir);
    wf_status st = write_raw(path, P->topography, n);
    if (st) return st;
    snprintf(path, sizeof(path), "%sNz_Y.bin", dir);
    FILE *f = fopen(path, "wb");
    if (!f) {
        wf::set_error("cannot create %s", path);
        return WF_ERR_IO;
    }
    const size_t w = fwrite(P->Nz_Y, sizeof(int), n, f);
    fclose(f);
    if (w != n) {
        wf::set_error("%s: short write", path);
        return WF_ERR_IO;
    }
    return WF_OK;
}

wf_status wf_save_fields(const Parameters *P, const char *dir, int n, const double *y, const double *pr)
{
    if (!P || !dir || !y || !pr) {
        wf::set_error("wf_save_fields: null argument");
        return WF_ERR_ARG;
    }
    const size_t N = (size_t)P->Nx * P->Ny * P->Nz, NY = (size_t)P->Nx * P->Ny * P->Nz_Y_max;
    const char *names[6] = {"u", "v", "w", "T", "Y", "p"};
    for (int q = 0; q < 6; q++) {
        char path[1024];
        snprintf(path, sizeof(path), "%s%s.bin.%d", dir, names[q], n);
        const double *src = (q < 5) ? y + q * N : pr;
        const wf_status st = write_raw(path, src, (q == 4) ? NY : N);
        if (st) return st;
    }
    return WF_OK;
}

}  // extern "C"
