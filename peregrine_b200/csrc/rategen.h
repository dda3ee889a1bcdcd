// The finite-rate source generated for one mechanism (rategen.cu): its CUDA
// source, and its compilation for sm_100a at a case's set-up.
#pragma once
#include <string>

#include "chem_types.h"
#include "physics.cuh"

namespace pgb {

// the source of the kernel pgb_gen_source for ns species and mechanism m
std::string rates_source(const Mech &m, const Species &sp, int ns);

// compiled for the sm_100a device: a cubin image, or false and the
// compiler's log (or why NVRTC could not be opened) in err
bool rates_compile(const std::string &src, std::string &cubin, std::string &err);

}  // namespace pgb
