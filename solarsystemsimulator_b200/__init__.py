"""B200-native (sm_100a) physics hot path of the SolarSystemSimulator.

Modules mirror the reference's backend modules and the film pipeline around
them; the compute runs in libsss.so (C ABI in include/sss.h, built by
build.py) and every module raises if that library or a GPU is missing:

  selfgrav_kernel  NBodySelfGrav: all-pairs self-gravity + tracers, KDK or
                   Yoshida-4, f64 or f32-pair/f64-accumulate
  nbody_kernel     NBodyCuda: few massive bodies + many asteroids (frame kernel)
  pm_kernel        NBodyPM and the 2-D isolated particle-mesh pieces
  broadphase       Erkennungskarte, bounce_hits, bounce_suche (colliding pairs)
  collide          CollisionResponse: merge sweep, bounce response, merges,
                   fragmentation
  ring             film ring slots and the self-gravity row reorder
  stream           StreamFrames: the server's per-sample cull, LOD, u16 frames
  batched          BatchedSystems: thousands of small systems per launch
  pm3d             3-D periodic PM, P3M pair term, learned correction + judge
  ewald            f64 Ewald direct sum (the judge of the 3-D PM)
  mlp              the correction network's weights, training and packing
  workloads        seeded synthetic inputs of the benchmark configurations
  replicas         max-over-ranks timing of independent replicas
"""
from ._lib import SSSError, load as load_library  # noqa: F401

__all__ = ["SSSError", "load_library"]
