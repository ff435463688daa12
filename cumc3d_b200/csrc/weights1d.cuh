// weights1d.cuh -- reconstruction weights of one cell of a 1D problem, shared
// by the host set-up of the batched engine (batch_host.cu) and the device
// set-up of the allocation-free entry point (noalloc.cu), so the two stay
// bit-identical by construction.  Both units compile without FMA contraction
// (--fmad=false on the device, -ffp-contract=off on the host).
//
// Formulas: PPM_WEIGHT / PPM_INTERPOLANT (solver/mhd/ppmc_module.f90:17-145),
// WENO_WEIGHT / WENO_INTERPOLANT (solver/mhd/weno_module.f90:35-149) and
// TVD_WEIGHT (solver/mhd/tvd_module.f90:25-55), in the same operation order as
// the 3D handle's build_weights.
#pragma once

namespace cumc {

// rec: 0..2 TVD, 3 PPM, 4 WENO.  dxr: cell widths of the padded row, dxr[j + 2]
// for j = -2..n+3.  w: the 14 weights of cell j (unused slots zero).
// Callers use j = 0..n+1 for PPM/WENO and j = -1..n+2 for TVD.
__host__ __device__ inline void batch_cell_weights(int rec, const double *dxr, int j, double *w) {
    for (int m = 0; m < 14; ++m) w[m] = 0.0;
    const double dm2 = (rec >= 3) ? dxr[j] : 0.0, dm1 = dxr[j + 1], dc = dxr[j + 2], dp1 = dxr[j + 3];
    const double dp2 = (rec >= 3) ? dxr[j + 4] : 0.0;
    if (rec == 4) {
        double a12 = dp2 / (dp1 + dp2), a01 = dp1 / (dc + dp1), a10 = dc / (dm1 + dc), a21 = dm1 / (dm2 + dm1);
        w[0] = (1.0 - a01); w[1] = a01; w[2] = (1.0 - a12); w[3] = a12; w[4] = (1.0 - a10);
        w[5] = a10; w[6] = (1.0 - a21); w[7] = a21; w[8] = (1.0 - a21); w[9] = a12;
    } else if (rec == 3) {
        double a1R = dc / (dc + dp1), a1L = dm1 / (dm1 + dc);
        double aR = 2.0 * dp1 * dc / (dp1 + dc), aL = 2.0 * dc * dm1 / (dc + dm1);
        double deltaXR = dm1 + dc + dp1 + dp2, deltaXL = dm2 + dm1 + dc + dp1;
        double z1R = (dm1 + dc) / (2.0 * dc + dp1), z1L = (dm2 + dm1) / (2.0 * dm1 + dc);
        double zR = (dp2 + dp1) / (2.0 * dp1 + dc), zL = (dp1 + dc) / (2.0 * dc + dm1);
        double cc1 = dc / (dm1 + dc + dp1), cp1 = dp1 / (dc + dp1 + dp2), cm1 = dm1 / (dm2 + dm1 + dc);
        double cc2 = (2.0 * dm1 + dc) / (dp1 + dc), cp2 = (2.0 * dc + dp1) / (dp2 + dp1), cm2 = (2.0 * dm2 + dm1) / (dc + dm1);
        double cc3 = (dc + 2.0 * dp1) / (dm1 + dc), cp3 = (dp1 + 2.0 * dp2) / (dc + dp1), cm3 = (dm1 + 2.0 * dc) / (dm2 + dm1);
        w[0] = a1L; w[1] = aL * (z1L - zL) / deltaXL; w[2] = (-dm1 * z1L) / deltaXL; w[3] = dc * zL / deltaXL;
        w[4] = a1R; w[5] = aR * (z1R - zR) / deltaXR; w[6] = (-dc * z1R) / deltaXR; w[7] = dp1 * zR / deltaXR;
        w[8] = cm1 * cm2; w[9] = cm1 * cm3; w[10] = cc1 * cc2; w[11] = cc1 * cc3; w[12] = cp1 * cp2; w[13] = cp1 * cp3;
    } else {
        w[0] = (dc + dp1) / dc;
        w[1] = (dc + dm1) / dc;
    }
}

}  // namespace cumc
