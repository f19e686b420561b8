/*
 * Files, statistics and prints of the reference's host program, restated so
 * that a run of the qcd2d driver leaves the same files as a run of kernel.cu:
 * names, headers, number formats and the Config_ binary layout are those of
 * functions/output.h:1-94, lattice_setup.h:83-100 and statistics.h:30-51
 * (they have to be alike for the files to be interchangeable).
 */
#ifndef QCD2D_REFIO_H
#define QCD2D_REFIO_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* the fields of `struct lattice` (lattice_setup.h:2-14) that the files print,
   for the full lattice */
typedef struct refio_lattice {
  int y, x, t, V, d;
  float beta, epsilon;
  int updates;
} refio_lattice;

/* statistics.h:30-39 (prints "%.10lf +- %.10lf\n" when print is set) */
void refio_mean_variance(const double* x, int n, double* results, int print);
/* statistics.h:41-51 (prints the first 10 lags) */
void refio_autocorrelation(const double* x, int n, int w, double mean, double variance, double* out);
/* statistics.h:17-28 on a host copy of the accept array */
double refio_mean_lattice_int(const int* accept, int n, const refio_lattice* l, int print);
/* lattice_setup.h:176-183 */
void refio_print_det(const double* phi, const refio_lattice* l);

/* output.h: each returns 0, or prints "Error creating the file" and returns 1
   (the reference calls exit(1) there; the driver does the same) */
int refio_save_autocorrelation(const char* dir, const double* r, int w, int n, int n_cor, int n_term,
                               const refio_lattice* l, const char* bound, const char* nsave, int av);
int refio_save_energy(const char* dir, double mean, double variance, int n_term, int n, int n_cor, double accept,
                      const refio_lattice* l, const char* bound, const char* nsave);
int refio_save_energy_av(const char* dir, double mean, double variance, double mean2, double variance2, int n_term,
                         int n, int n_cor, double accept, const refio_lattice* l, const char* bound,
                         const char* nsave);
int refio_save_en_seq(const char* dir, const double* plaq, const double* energy, int n_term, int n, int n_cor,
                      double accept, const refio_lattice* l, const char* bound, const char* nsave);
int refio_save_conf(const char* dir, const double* phi, const refio_lattice* l, int n_term, int init,
                    const char* bound, const char* nsave);
/* lattice_setup.h:83-100, with the size checked: returns 1 (after the
   reference's message) when a file is missing, short or malformed */
int refio_read_conf(const char* dir, double* phi, const refio_lattice* l, int* n_term, int* init, const char* bound,
                    const char* nsave);

#ifdef __cplusplus
}
#endif
#endif
