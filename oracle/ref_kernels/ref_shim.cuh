/*
 * The reference's 2D kernel files use BDIMX, BDIMY, radius (and the *2
 * variants) without defining them anywhere in its tree.  The values below are
 * inferred from the constants the same files do define (BDIMX1 = 32,
 * BDIMY1 = 16, radius1 = 6 in elastic_2D_kernel_2.cu:1-3; the same in
 * elastic_2D_kernel_3.cu:1-3) — an inference, recorded as such.
 */
#pragma once
#define BDIMX 32
#define BDIMY 16
#define radius 6
#define BDIMX2 32
#define BDIMY2 16
#define radius2 6
