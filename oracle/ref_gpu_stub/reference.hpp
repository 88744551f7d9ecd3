// Stand-in for the reference's src/reference.hpp when its GPU distance kernel
// (src/gpu/dist.cu) is compiled on its own by oracle/Makefile.  The kernel and
// the launch helpers used by oracle/ref_gpu_dists.cu need only the name of the
// sketch container; its Eigen- and HDF5-backed definition is not built.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

class Reference {};
