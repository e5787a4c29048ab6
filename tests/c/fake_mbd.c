/* Stand-in for libmbd_b200.so with the entry points the pmbd_b200
 * executable calls, so that its host logic runs on a machine without a GPU
 * (tests/test_host_cpp.py links the executable against this file built as
 * libmbd_b200.so).  It computes nothing:
 *   FAKE_MBD_VALUES  file of hex floats: energy c6_mol nimag sc1 sc2 sc3,
 *                    c6_eff[N], alpha_eff[N], molpol_eig[63], omega[21];
 *                    mbd_rsscs_energy returns them, mbd_rsscs_frequency_grid
 *                    the omegas;
 *   FAKE_MBD_STATUS  status mbd_rsscs_energy returns instead (optional);
 *   FAKE_MBD_RECORD  file that receives every argument the executable
 *                    passed: the mbd_geom fields, the mode, the network
 *                    switch and the parameters it set.
 * mbd_rsscs_energy_batch runs mbd_rsscs_energy on each geometry in turn. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mbd_b200.h"

struct mbd_ctx {
    int device;
};

static const char* kSymbols[] = {
    "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",  "S",  "Cl", "Ar",
    "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr",
    "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe"};

static FILE* record(void) {
    const char* p = getenv("FAKE_MBD_RECORD");
    return p ? fopen(p, "a") : NULL;
}

int mbd_rsscs_element_z(const char* symbol) {
    for (size_t k = 0; k < sizeof(kSymbols) / sizeof(kSymbols[0]); ++k)
        if (strcmp(symbol, kSymbols[k]) == 0) return (int)k + 1;
    return 0;
}

const char* mbd_rsscs_strerror(int code) { return code == MBD_ERR_UNKNOWN_ELEMENT ? "fake: unknown element" : "fake error"; }

static int read_values(double* v, int count) {
    const char* p = getenv("FAKE_MBD_VALUES");
    FILE* f = p ? fopen(p, "r") : NULL;
    if (!f) return 0;
    int k = 0;
    char tok[128];
    while (k < count && fscanf(f, "%127s", tok) == 1) v[k++] = strtod(tok, NULL);
    fclose(f);
    return k;
}

int mbd_rsscs_create(mbd_ctx** ctx, int device) {
    *ctx = (mbd_ctx*)malloc(sizeof(mbd_ctx));
    (*ctx)->device = device;
    FILE* r = record();
    if (r) {
        fprintf(r, "device %d\n", device);
        fclose(r);
    }
    return MBD_OK;
}

void mbd_rsscs_destroy(mbd_ctx* ctx) { free(ctx); }

int mbd_rsscs_learned_param_count(void) { return 16274; }

int mbd_rsscs_learned_use_network(mbd_ctx* ctx, int on) {
    (void)ctx;
    FILE* r = record();
    if (r) {
        fprintf(r, "use_network %d\n", on);
        fclose(r);
    }
    return MBD_OK;
}

int mbd_rsscs_learned_set_params(mbd_ctx* ctx, const float* params, int n) {
    (void)ctx;
    FILE* r = record();
    if (r) {
        double sum = 0.0;
        for (int i = 0; i < n; ++i) sum += (double)params[i] * (double)(i % 7 + 1);
        fprintf(r, "set_params %d %a\n", n, sum);
        fclose(r);
    }
    return MBD_OK;
}

int mbd_rsscs_frequency_grid(double* omega, double* weight, int n) {
    if (n < MBD_N_FREQ) return MBD_ERR_ARG;
    /* the omegas are the last 21 values of the file; count them from the end */
    static double v[1 << 16];
    const int k = read_values(v, 1 << 16);
    if (k < MBD_N_FREQ) return MBD_ERR_ARG;
    for (int f = 0; f < MBD_N_FREQ; ++f) {
        omega[f] = v[k - MBD_N_FREQ + f];
        if (weight) weight[f] = 0.0;
    }
    return MBD_OK;
}

int mbd_rsscs_energy(mbd_ctx* ctx, const mbd_geom* g, int mode, mbd_result* out) {
    (void)ctx;
    FILE* r = record();
    if (r) {
        fprintf(r, "mode %d\nn_atoms %d\nn_periodic %d\nxc %d\n", mode, g->n_atoms, g->n_periodic, g->xc);
        fprintf(r, "cuts %a %a %a\nvacuum %d %d %d\n", g->scs_cut_A, g->cfdm_cut_A, g->sc_cut_A, g->vacuum[0],
                g->vacuum[1], g->vacuum[2]);
        for (int i = 0; i < g->n_atoms; ++i)
            fprintf(r, "atom %d %a %a %a %a\n", g->z[i], g->coords_bohr[3 * i], g->coords_bohr[3 * i + 1],
                    g->coords_bohr[3 * i + 2], g->hirshfeld[i]);
        for (int i = 0; i < 9; ++i) fprintf(r, "lattice %a\n", g->lattice_bohr ? g->lattice_bohr[i] : 0.0);
        fclose(r);
    }
    const char* fs = getenv("FAKE_MBD_STATUS");
    if (fs && atoi(fs) != 0) {
        out->status = atoi(fs);
        return out->status;
    }
    for (int i = 0; i < g->n_atoms; ++i)
        if (g->z[i] == 0) return out->status = MBD_ERR_UNKNOWN_ELEMENT;
    const int N = g->n_atoms;
    static double v[1 << 16];
    if (read_values(v, 1 << 16) < 6 + 2 * N + 63) return out->status = MBD_ERR_ARG;
    out->energy_Ha = v[0];
    out->c6_mol = v[1];
    out->nimag = (int)v[2];
    for (int k = 0; k < 3; ++k) out->supercell[k] = (int)v[3 + k];
    for (int i = 0; i < N; ++i) {
        if (out->c6_eff) out->c6_eff[i] = v[6 + i];
        if (out->alpha_eff) out->alpha_eff[i] = v[6 + N + i];
    }
    if (out->molpol_eig)
        for (int k = 0; k < 63; ++k) out->molpol_eig[k] = v[6 + 2 * N + k];
    out->status = MBD_OK;
    return MBD_OK;
}

int mbd_rsscs_energy_batch(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms, int mode, mbd_result* out) {
    int first = MBD_OK;
    for (int g = 0; g < n_geom; ++g) {
        const int st = mbd_rsscs_energy(ctx, &geoms[g], mode, &out[g]);
        if (st != MBD_OK && first == MBD_OK) first = st;
    }
    return first;
}
