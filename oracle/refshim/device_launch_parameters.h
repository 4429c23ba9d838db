// Host-compilation shim (test infrastructure only): the CUDA header of the
// same name is not needed when the reference kernels run on the host.
#pragma once
