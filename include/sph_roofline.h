/*
 * sph_roofline.h - algorithmic bytes of the WCSPH step, per particle-step.
 *
 * FP32 SoA fields, each moved once per stage; neighbour reads are assumed
 * to hit in cache (they are counted separately as pair work). The stage
 * figures add up to 408 B per particle-step. The five CUDA kernels of a step
 * each own a subset of the stages (right-hand column).
 *
 *   stage                                bytes   kernel
 *   kick 1 (v, a in; v out)                 36   xsph_drift
 *   XSPH (x, v, m, rho in; dv out)          44   xsph_drift
 *   drift + clamp (x, v, dv in; x, v out)   60   xsph_drift
 *   binning (x in; key out)                 16   xsph_drift
 *   counting-sort scatter                    8   sort (fill + reorder)
 *   SoA reorder (x,v,a,rho,p,m,id rw; perm) 108  sort
 *   density + delta-SPH + EOS               28   density
 *   forces                                  48   forces
 *   kick 2                                  36   forces
 *   dt reduction                            24   forces
 *   plus per grid cell: counts + offsets     8   sort (scan)
 *   plus per boundary particle: x,m in, p out 20  boundary_pressure (Adami)
 */
#ifndef SPH_ROOFLINE_H
#define SPH_ROOFLINE_H

#define SPH_BYTES_PER_PARTICLE_STEP 408
#define SPH_BYTES_XSPH_DRIFT 156
#define SPH_BYTES_SORT 116
#define SPH_BYTES_DENSITY 28
#define SPH_BYTES_FORCES 108
#define SPH_BYTES_PER_CELL 8
#define SPH_BYTES_PER_BOUNDARY 20

/*
 * FP32 operations of the pair work, counted from the kernels' expressions
 * (every IEEE add, subtract, multiply, compare, divide and square root counts
 * one; --fmad=false forms no FMA). The neighbour kernels are bound by
 * instruction issue, not by HBM, so their roofline is this count against
 * the FP32 peak: 128 lanes per SM x 148 SMs x the SM clock.
 *
 *   candidate test of the 27-cell scan: 3 sub, 3 mul, 2 add, 1 compare     9
 *     (per particle of the 27 cells, as the reference's neighbour loop
 *     tests them, neighbor.rs:129-182)
 *   density interaction: distance 8, sqrt 1, gradient 17, r.gradW 5,
 *     density difference 1, delta-SPH term 6, W 10, rho += m W 2           50
 *   forces interaction: distance 8, sqrt 1, gradient 17, pressure factor 3,
 *     pressure sum 6, dv 3, v.r 5, compare 1, viscous term 18 (evaluated
 *     for every pair, a receding one adding a signed zero)                 62
 *   XSPH interaction: distance 8, sqrt 1, W 10, rho avg 2, factor 3,
 *     velocity sum 9                                                       33
 */
#define SPH_FLOPS_SCAN_PER_CANDIDATE 9
#define SPH_FLOPS_DENSITY_PER_INTERACTION 50
#define SPH_FLOPS_FORCES_PER_INTERACTION 62
#define SPH_FLOPS_XSPH_PER_INTERACTION 33
#define SPH_FP32_LANES_PER_SM 128
#define SPH_SM_COUNT 148

#endif
