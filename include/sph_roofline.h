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

#endif
