"""B200-native CAFFE hot path: SIMPLE / PISO / IB-PISO finite-volume iteration on
structured hexahedral meshes, with the per-iteration work in hand-written sm_100a
CUDA kernels behind a C ABI (include/caffe_b200.h)."""
