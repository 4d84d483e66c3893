/*
 * sg_workload.h -- the prescribed Eulerian velocity of the time-stepped
 * benchmark.  No counterpart in the reference, whose velocity comes from its
 * flow solver: this generates the synthetic flow that the advection runs
 * (capsules moved by the interpolated velocity) are driven by, on the GPU,
 * so that a step needs no host work.
 */
#ifndef SG_WORKLOAD_H
#define SG_WORKLOAD_H
#ifdef __cplusplus
extern "C" {
#endif

#define SG_FLOW_MAX_MODES 32

/* u, v, w on the staggered grid including the one-cell halo, arrays of
 * (ktot+2) x (jtot+2) x (itot+2) with x fastest (the Eulerian layout of
 * sg_coupling.h), at the time *t (a device address, read when the work runs,
 * so that a captured CUDA graph can advance it):
 *   u_c = sum_q amp[q][c] cos(2 pi nx_q x / Lx + 2 pi ny_q y / Ly
 *                             + phase_q + omega_q t) sin(pi z / Lz)
 * with (x, y, z) the location of component c (face i dx along its own
 * direction, centre (i - 1/2) dx along the others) and L = (itot dx, jtot dy,
 * ktot dz); u additionally gets shear * z.  Evaluated in FP64 and rounded
 * once to the output type (fp32 != 0: float arrays, else double).  Rows of up
 * to 1024 cells: itot + 2 <= 1024.  nmodes <=
 * SG_FLOW_MAX_MODES; the mode arrays are host memory (nmodes each, amp
 * nmodes x 3), copied into the launch.  `work` is device scratch of
 * 3 (jtot+2)(itot+2) doubles.  Queued on `stream`; returns 0, or SG_ERR_ARG
 * (bad sizes or pointers) or SG_ERR_CUDA (codes of sg_coupling.h). */
int sg_prescribed_flow(int itot, int jtot, int ktot, double dx, double dy, double dz, int nmodes, const double* nx,
                       const double* ny, const double* phase, const double* amp, const double* omega, double shear,
                       const double* t, int fp32, void* u, void* v, void* w, void* work, void* stream);

#ifdef __cplusplus
}
#endif
#endif
