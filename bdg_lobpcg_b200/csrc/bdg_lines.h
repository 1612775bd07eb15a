// bdg_lines.h -- FFT pass kernels with register-resident line transforms
// (bdg_lines.cu).  Internal to the library.
#pragma once

#include "bdg_dev.h"
#include "bdg_kern.cuh"

// Line lengths the register kernels cover.
bool bdgd_lines_size_ok(int n);

// Whether the register pass kernels can run program p on context c (3D/2D
// grids of supported line lengths; real fields also need an even number of
// x rows, which are transformed in pairs).
bool bdgd_lines_usable(const bdgd_ctx *c, const Prog &p);

// Full operator apply (forward passes, k-space multiply, inverse passes,
// epilogue) of program p on nc columns.  spec holds nc * p.J spectra.
int bdgd_lines_apply(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, int prec, const void *x, long long ldx,
                     void *y, long long ldy, void *spec, int nc);
