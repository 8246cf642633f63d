"""CPU restatement of the viewer's Frame message (test infrastructure only).

``build_frame`` follows server/src/ws.rs:233-290: tag 0x02, frame number
(u64), subsampled particle count (u32), simulation time (f64), then for
every stride-th particle (original order) x, y, z, temperature (f32), fluid
type (u8), density ratio (u16: (density / rest density) * 1000 in f32,
clamped to [0, 65535], truncated; NaN gives 0), a zero byte; little endian.
"""
from __future__ import annotations

import struct

import numpy as np

WATER_REST_DENSITY = np.float32(1000.0)  # kernel/src/eos.rs:7
AIR_REST_DENSITY = np.float32(1.204)     # kernel/src/eos.rs:10


def density_ratio(density, fluid_type) -> np.ndarray:
    rest = np.where(np.asarray(fluid_type) == 0, WATER_REST_DENSITY, AIR_REST_DENSITY).astype(np.float32)
    with np.errstate(invalid="ignore", over="ignore", divide="ignore"):
        r = (np.asarray(density, np.float32) / rest).astype(np.float32) * np.float32(1000.0)
        r = np.where(np.isnan(r), np.float32(0.0), np.clip(r, np.float32(0.0), np.float32(65535.0)))
    return np.trunc(r).astype(np.uint16)


def build_frame(particles, subsample_count: int, frame_number: int, sim_time: float) -> bytes:
    n = len(particles.x)
    stride = max(n // subsample_count, 1) if subsample_count > 0 else 1
    count = min(n // stride, subsample_count)
    out = bytearray(struct.pack("<BQId", 0x02, frame_number, count, sim_time))
    idx = np.arange(0, n, stride)[:count]
    ratio = density_ratio(particles.density[idx], particles.fluid_type[idx])
    for k, i in enumerate(idx):
        out += struct.pack("<ffffBHB", float(particles.x[i]), float(particles.y[i]), float(particles.z[i]),
                           float(particles.temperature[i]), int(particles.fluid_type[i]), int(ratio[k]), 0)
    return bytes(out)
