"""The FLIP particle record.

Same 40-byte layout as the reference's ``ivock::particle``
(Smoke_Solver/fluid_particle.h:14-20): pos f32x3, vel f32x3, dens, temp,
hash_idx, sub_hash_idx.  The transfer kernels read pos/vel straight out of an
array of these records, so a caller's particle vector can be handed over
without repacking.
"""
import numpy as np

PARTICLE_DTYPE = np.dtype([("pos", "<f4", (3,)), ("vel", "<f4", (3,)), ("dens", "<f4"), ("temp", "<f4"),
                           ("hash_idx", "<i4"), ("sub_hash_idx", "<i4")])
assert PARTICLE_DTYPE.itemsize == 40
PARTICLE_BYTES = 40
