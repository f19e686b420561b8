/* Reference-compatible files, statistics and prints (see refio.h). */
#include "refio.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static void path(char* out, size_t cap, const char* dir, const char* name) {
  if (dir && dir[0])
    snprintf(out, cap, "%s/%s", dir, name);
  else
    snprintf(out, cap, "%s", name);
}

/* the name stem shared by every output: <kind>_<t>_<x>_<y>_B_<beta>_<bc>_<n> */
static void stem(char* out, size_t cap, const char* kind, const refio_lattice* l, const char* bound,
                 const char* nsave, const char* suffix) {
  snprintf(out, cap, "%s_%d_%d_%d_B_%.2lf_%s_%s%s", kind, l->t, l->x, l->y, (double)l->beta, bound, nsave, suffix);
}

static FILE* open_out(const char* dir, const char* name, const char* mode) {
  char p[1024];
  path(p, sizeof(p), dir, name);
  FILE* f = fopen(p, mode);
  if (!f) printf("Error creating the file");
  return f;
}

void refio_mean_variance(const double* x, int n, double* results, int print) {
  double s = 0, s2 = 0;
  for (int i = 0; i < n; i++) {
    s += x[i];
    s2 += x[i] * x[i];
  }
  results[0] = s / n;
  results[1] = (s2 / n - results[0] * results[0]);
  if (print) printf("%.10lf +- %.10lf\n", results[0], sqrt(results[1] / (n - 1)));
}

void refio_autocorrelation(const double* x, int n, int w, double mean, double variance, double* out) {
  for (int lag = 1; lag < w + 1; lag++) {
    double s = 0;
    for (int j = 0; j < n - lag; j++) s += (x[j] - mean) * (x[j + lag] - mean);
    out[lag - 1] = s / (n - lag) / variance;
    if (lag < 11) printf("%d %lf\n", lag, out[lag - 1]);
  }
}

double refio_mean_lattice_int(const int* accept, int n, const refio_lattice* l, int print) {
  double mean = 0, variance = 0;
  for (int i = 0; i < l->V; i++) {
    mean += accept[i];
    variance += (double)accept[i] * accept[i];
  }
  mean = mean / l->V / n;
  variance = sqrt((variance / l->V / n - mean * mean) / l->V / (n - 1));
  if (print) printf("%.10lf +- %.10lf\n", mean, variance);
  return mean;
}

void refio_print_det(const double* phi, const refio_lattice* l) {
  double det = 0;
  for (long long i = 0; i < (long long)l->V * l->d; i++) {
    const double* a = phi + i * 4;
    det += a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
  }
  printf("Av det %.16lf\n", det / l->V / l->d);
}

int refio_save_autocorrelation(const char* dir, const double* r, int w, int n, int n_cor, int n_term,
                               const refio_lattice* l, const char* bound, const char* nsave, int av) {
  char name[512];
  stem(name, sizeof(name), av ? "Autocorrelation_av" : "Autocorrelation", l, bound, nsave, ".txt");
  FILE* f = open_out(dir, name, "w");
  if (!f) return 1;
  fprintf(f, "N_termalizacion %d N %d N_correlation %d  D_t %d D_x %d D_ y %d beta %.2lf deltaphi %.2lf\n", n_term,
          n, n_cor, l->t, l->x, l->y, (double)l->beta, (double)l->epsilon);
  fprintf(f, "N Autocorrelation\n");
  for (int i = 0; i < w; i++) fprintf(f, "%d %.10lf\n", i + 1, r[i]);
  fclose(f);
  return 0;
}

int refio_save_energy(const char* dir, double mean, double variance, int n_term, int n, int n_cor, double accept,
                      const refio_lattice* l, const char* bound, const char* nsave) {
  char name[512];
  stem(name, sizeof(name), "Energy", l, bound, nsave, ".txt");
  FILE* f = open_out(dir, name, "w");
  if (!f) return 1;
  fprintf(f, "N_termalizacion %d N %d N_correlation %d  D_t %d D_x %d D_ y %d deltaphi %.2lf accept %.2lf\n", n_term,
          n, n_cor, l->t, l->x, l->y, (double)l->epsilon, accept);
  fprintf(f, "M Energy Error\n");
  fprintf(f, "%f %.10lf %.10lf\n", (double)l->beta, mean, sqrt(variance / (n - 1)));
  fclose(f);
  return 0;
}

int refio_save_energy_av(const char* dir, double mean, double variance, double mean2, double variance2, int n_term,
                         int n, int n_cor, double accept, const refio_lattice* l, const char* bound,
                         const char* nsave) {
  char name[512];
  stem(name, sizeof(name), "Energy_av", l, bound, nsave, ".txt");
  FILE* f = open_out(dir, name, "w");
  if (!f) return 1;
  fprintf(f,
          "N_termalizacion %d N %d N_correlation %d N_updates %d  D_t %d D_x %d D_ y %d deltaphi %.2lf accept %.2lf\n",
          n_term, n, n_cor, l->updates, l->t, l->x, l->y, (double)l->epsilon, accept);
  fprintf(f, "M Energy/Avplaquette Error\n");
  fprintf(f, "%f %.10lf %.10lf\n", (double)l->beta, mean, sqrt(variance / (n - 1)));
  fprintf(f, "%f %.10lf %.10lf\n", (double)l->beta, mean2, sqrt(variance2 / (n - 1)));
  fclose(f);
  return 0;
}

int refio_save_en_seq(const char* dir, const double* plaq, const double* energy, int n_term, int n, int n_cor,
                      double accept, const refio_lattice* l, const char* bound, const char* nsave) {
  char name[512];
  stem(name, sizeof(name), "Check", l, bound, nsave, ".txt");
  FILE* f = open_out(dir, name, "w");
  if (!f) return 1;
  fprintf(f,
          "N_termalizacion %d N %d N_correlation %d N_updates %d  D_t %d D_x %d D_y %d deltaphi %.2lf accept %.2lf\n",
          n_term, n, n_cor, l->updates, l->t, l->x, l->y, (double)l->epsilon, accept);
  fprintf(f, "I Energy Avpl\n");
  for (int i = 0; i < n; i++) fprintf(f, "%d %.10lf %.10lf\n", i, energy[i], plaq[i]);
  fclose(f);
  return 0;
}

int refio_save_conf(const char* dir, const double* phi, const refio_lattice* l, int n_term, int init,
                    const char* bound, const char* nsave) {
  char name[512];
  stem(name, sizeof(name), "Config", l, bound, nsave, ".txt");
  FILE* f = open_out(dir, name, "wb");
  if (!f) return 1;
  const size_t n = (size_t)l->V * 12;
  if (fwrite(phi, sizeof(double), n, f) != n) {
    fclose(f);
    printf("Error creating the file");
    return 1;
  }
  fclose(f);
  stem(name, sizeof(name), "Config", l, bound, nsave, "_data.txt");
  f = open_out(dir, name, "w");
  if (!f) return 1;
  fprintf(f, "N_termalization %d Type_termalization %d", n_term, init);
  fclose(f);
  return 0;
}

int refio_read_conf(const char* dir, double* phi, const refio_lattice* l, int* n_term, int* init, const char* bound,
                    const char* nsave) {
  char name[512], p[1024];
  stem(name, sizeof(name), "Config", l, bound, nsave, ".txt");
  path(p, sizeof(p), dir, name);
  FILE* f = fopen(p, "rb");
  if (!f) {
    printf("Error creating the file");
    return 1;
  }
  const size_t n = (size_t)l->V * 12;
  size_t got = fread(phi, sizeof(double), n, f);
  int extra = fgetc(f);
  fclose(f);
  if (got != n || extra != EOF) {
    printf("Error reading %s: %zu of %zu doubles%s\n", p, got, n, extra != EOF ? " and trailing bytes" : "");
    return 1;
  }
  stem(name, sizeof(name), "Config", l, bound, nsave, "_data.txt");
  path(p, sizeof(p), dir, name);
  f = fopen(p, "r");
  if (!f) {
    printf("Error creating the file");
    return 1;
  }
  int ok = fscanf(f, "N_termalization %d Type_termalization %d", n_term, init);
  fclose(f);
  if (ok != 2) {
    printf("Error reading %s\n", p);
    return 1;
  }
  return 0;
}
