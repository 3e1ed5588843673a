// Small host helpers shared by the app-layer sources: CUDA and library status checks
// turned into the reference's exception types, and uint32 index lists uploaded to
// the device.
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "troy_b200.hpp"

namespace troyn {
namespace detail {

inline void cuda_ok(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

inline void tb_ok(int st) {
    if (st == TB_OK) return;
    if (st == TB_ERR_INVALID_ARGUMENT) throw std::invalid_argument(tb_last_error());
    if (st == TB_ERR_UNSUPPORTED) throw std::logic_error(tb_last_error());
    throw std::runtime_error(tb_last_error());
}

// uint32 arrays travel packed two per device word.
inline DeviceBuffer upload_u32(const std::vector<std::uint32_t> &v) {
    std::vector<std::uint64_t> w((v.size() + 1) / 2, 0);
    if (!v.empty()) std::memcpy(w.data(), v.data(), v.size() * 4);
    DeviceBuffer b;
    b.fromHost(w.data(), w.size());
    return b;
}

}  // namespace detail
}  // namespace troyn
