/*
 * bdg_io.c -- text I/O with the formats and return codes of the reference
 * (pstuermer/BDG_LOBPCG src/io.c:13-165): wavefunction as one "re im" pair
 * per line; eigenvalues appended as one tab-separated "%.8e" row; modes as
 * "re<TAB>im" pairs, one grid row per line, a blank line between 2D rows /
 * 3D slices.
 */
#include <stdarg.h>
#include <string.h>

#include "bdg/bdg_internal.h"

int bdg_load_wavefunction(bdg_t *bdg, const char *filename) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_load_wavefunction");
  const uint64_t size = bdg->ctx->size;
  FILE *f = fopen(filename, "r");
  if (f == NULL) return -1;
  const int cplx = bdg->complex_psi0;
  f64 *buf = xcalloc(size, cplx ? sizeof(c64) : sizeof(f64));
  for (uint64_t i = 0; i < size; i++) {
    f64 re, im;
    if (fscanf(f, "%lf %lf", &re, &im) != 2) {
      safe_free((void **)&buf);
      fclose(f);
      return -2;
    }
    if (cplx) {
      buf[2 * i] = re;
      buf[2 * i + 1] = im;
    } else {
      buf[i] = re;
    }
  }
  fclose(f);
  bdg_set_wavefunction(bdg, buf, size);
  safe_free((void **)&buf);
  return 0;
}

int bdg_load_wavefunction_fmt(bdg_t *bdg, const char *fmt, ...) {
  char name[512];
  va_list ap;
  va_start(ap, fmt);
  const int n = vsnprintf(name, sizeof name, fmt, ap);
  va_end(ap);
  if (n < 0 || (size_t)n >= sizeof name) return -1;
  return bdg_load_wavefunction(bdg, name);
}

int bdg_write_eigenvalues(const bdg_t *bdg, const char *filename) {
  if (bdg->eigvals == NULL) return -3;
  FILE *f = fopen(filename, "a");
  if (f == NULL) return -1;
  for (uint64_t i = 0; i < bdg->nev; i++) {
    fprintf(f, "%.8e", bdg->eigvals[i]);
    if (i + 1 < bdg->nev) fputc('\t', f);
  }
  fputc('\n', f);
  fclose(f);
  return 0;
}

static int write_mode(const bdg_t *bdg, uint64_t idx, const void *modes, const char *basename, const char *part) {
  if (modes == NULL) return -3;
  if (idx >= bdg->nev) return -2;
  char name[512];
  snprintf(name, sizeof name, "%s_%s_%lu.dat", basename, part, (unsigned long)idx);
  FILE *f = fopen(name, "w");
  if (f == NULL) return -1;
  const matmul_ctx_t *ctx = bdg->ctx;
  const uint64_t size = ctx->size, dim = ctx->dim;
  const uint64_t Nx = ctx->N[0];
  const uint64_t Ny = dim > 1 ? ctx->N[1] : 1;
  const uint64_t Nz = dim > 2 ? ctx->N[2] : 1;
  const int cplx = bdg->complex_psi0;
  const f64 *md = (const f64 *)modes + idx * size * (cplx ? 2 : 1);
  for (uint64_t k = 0; k < Nz; k++) {
    for (uint64_t j = 0; j < Ny; j++) {
      for (uint64_t i = 0; i < Nx; i++) {
        const uint64_t p = (k * Ny + j) * Nx + i;
        const f64 re = cplx ? md[2 * p] : md[p];
        const f64 im = cplx ? md[2 * p + 1] : 0.0;
        fprintf(f, "%.8e\t%.8e", re, im);
        if (dim == 1) {
          fputc('\n', f);
        } else if (i + 1 < Nx) {
          fputc('\t', f);
        }
      }
      if (dim >= 2) fputc('\n', f);
      if (dim == 2 && j + 1 < Ny) fputc('\n', f);
    }
    if (dim == 3 && k + 1 < Nz) fputc('\n', f);
  }
  fclose(f);
  return 0;
}

int bdg_write_mode_u(const bdg_t *bdg, uint64_t mode_idx, const char *basename) {
  return write_mode(bdg, mode_idx, bdg->modes_u, basename, "u");
}

int bdg_write_mode_v(const bdg_t *bdg, uint64_t mode_idx, const char *basename) {
  return write_mode(bdg, mode_idx, bdg->modes_v, basename, "v");
}

/* ---- binary formats (no counterpart in the reference) -----------------------
 * The reference's text files keep 8 significant digits and cost one fprintf
 * per value (about 40 MB and seconds per mode at 128^3).  These files hold
 * the exact doubles: a 64-byte header (bdg_bin_header_t, bdg/bdg_b200.h) and
 * `count` consecutive fields of the grid's `size` values (f64, or interleaved
 * re, im for c128), x fastest, in the host's byte order. */
static int bin_write(const char *filename, const bdg_t *bdg, uint32_t kind, uint32_t dtype, uint64_t count,
                     uint64_t per, const void *data) {
  if (data == NULL) return -3;
  FILE *f = fopen(filename, "wb");
  if (f == NULL) return -1;
  bdg_bin_header_t h;
  memset(&h, 0, sizeof h);
  memcpy(h.magic, BDG_BIN_MAGIC, 8);
  h.version = BDG_BIN_VERSION;
  h.kind = kind;
  h.dtype = dtype;
  h.dim = (uint32_t)bdg->ctx->dim;
  for (uint64_t d = 0; d < 3; d++) h.N[d] = d < bdg->ctx->dim ? bdg->ctx->N[d] : 1;
  h.count = count;
  const size_t esz = dtype == BDG_BIN_C128 ? 2 * sizeof(f64) : sizeof(f64);
  const size_t nel = (size_t)(count * per);
  int rc = 0;
  if (fwrite(&h, sizeof h, 1, f) != 1 || (nel && fwrite(data, esz, nel, f) != nel)) rc = -1;
  if (fclose(f) != 0) rc = -1;
  return rc;
}

int bdg_write_wavefunction_bin(const bdg_t *bdg, const char *filename) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_write_wavefunction_bin");
  const int cplx = bdg->complex_psi0;
  return bin_write(filename, bdg, BDG_BIN_WAVEFUNCTION, cplx ? BDG_BIN_C128 : BDG_BIN_F64, 1, bdg->ctx->size,
                   bdg->ctx->wf);
}

int bdg_write_modes_bin(const bdg_t *bdg, int part, const char *filename) {
  if (part != 0 && part != 1) return -2;
  if (bdg->ctx == NULL) return -3;
  const int cplx = bdg->complex_psi0;
  return bin_write(filename, bdg, part ? BDG_BIN_MODES_V : BDG_BIN_MODES_U, cplx ? BDG_BIN_C128 : BDG_BIN_F64,
                   bdg->nev, bdg->ctx->size, part ? bdg->modes_v : bdg->modes_u);
}

int bdg_write_eigenvalues_bin(const bdg_t *bdg, const char *filename) {
  if (bdg->eigvals == NULL || bdg->ctx == NULL) return -3;
  return bin_write(filename, bdg, BDG_BIN_EIGENVALUES, BDG_BIN_F64, bdg->nev, 1, bdg->eigvals);
}

int bdg_load_wavefunction_bin(bdg_t *bdg, const char *filename) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_load_wavefunction_bin");
  FILE *f = fopen(filename, "rb");
  if (f == NULL) return -1;
  bdg_bin_header_t h;
  const matmul_ctx_t *ctx = bdg->ctx;
  const int cplx = bdg->complex_psi0;
  int ok = fread(&h, sizeof h, 1, f) == 1 && memcmp(h.magic, BDG_BIN_MAGIC, 8) == 0 &&
           h.version == BDG_BIN_VERSION && h.kind == BDG_BIN_WAVEFUNCTION && h.count == 1 &&
           h.dtype == (uint32_t)(cplx ? BDG_BIN_C128 : BDG_BIN_F64) && h.dim == (uint32_t)ctx->dim;
  for (uint64_t d = 0; ok && d < 3; d++) ok = h.N[d] == (d < ctx->dim ? ctx->N[d] : 1);
  if (!ok) {
    fclose(f);
    return -2;
  }
  const size_t esz = cplx ? 2 * sizeof(f64) : sizeof(f64);
  void *buf = xcalloc(ctx->size, esz);
  const int full = fread(buf, esz, ctx->size, f) == ctx->size;
  fclose(f);
  if (!full) {
    safe_free(&buf);
    return -2;
  }
  bdg_set_wavefunction(bdg, buf, ctx->size);
  safe_free(&buf);
  return 0;
}
