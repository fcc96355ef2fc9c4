"""B200-native MPS time-step hot path: the reference's C entry points over hand-written
sm_100a CUDA kernels (libmps_b200.so, libmps3d.so, libmps2d.so), with a ctypes session
layer, workload builders and a differentiable rollout."""
