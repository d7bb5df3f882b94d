"""B200-native (sm_100a) collision-and-dynamics hot path with the data
contracts of ReactPhysics3D's narrow phase (NarrowPhaseInfoBatch) behind a
C ABI (include/rp3dg.h, reactphysics3d_b200/_lib/librp3dg.so)."""
