// sfgpu_batch_wide.cu -- the wide instantiation of the batched kernel (the
// twelve-neighbour 3D lattice types and the force ensemble), in a
// translation unit of its own.
#include "sfgpu_batch_kernel.cuh"

BatchKernel batch_kernel_wide() { return batch_diis_kernel_t<true>; }
