// Drop-in for the reference's include/LinAlg/linalg.hpp: the LinAlg types.
#ifndef MFGPU_LINALG_HPP
#define MFGPU_LINALG_HPP 1
#include "vec.hpp"
#include "dense.hpp"
#include "sparse.hpp"
#endif
