// Command-line helpers shared by the example binaries (the reference's Cli.hpp / PhotonCli.hpp
// value rules): unsigned integers without sign or trailing characters and with overflow checks,
// finite doubles, enumerated words; malformed values throw std::invalid_argument, which the
// binaries turn into exit code 2 with the usage text.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <initializer_list>
#include <limits>
#include <stdexcept>
#include <string>
#include <string_view>

#include "graphflow_b200.h"

namespace gfcli {

inline std::uint64_t parseU64(std::string_view flag, const std::string& value)
{
    if (value.empty() || value.find_first_not_of("0123456789") != std::string::npos)
        throw std::invalid_argument(std::string(flag) + ": expected an unsigned integer, got '" + value + "'");
    std::uint64_t v = 0u;
    for (const char ch : value) {
        const std::uint64_t d = static_cast<std::uint64_t>(ch - '0');
        if (v > (std::numeric_limits<std::uint64_t>::max() - d) / 10u)
            throw std::invalid_argument(std::string(flag) + ": value '" + value + "' exceeds 64 bits");
        v = v * 10u + d;
    }
    return v;
}

inline std::uint32_t parseU32(std::string_view flag, const std::string& value, bool allowZero = false)
{
    const std::uint64_t v = parseU64(flag, value);
    if (v > std::numeric_limits<std::uint32_t>::max())
        throw std::invalid_argument(std::string(flag) + ": value '" + value + "' exceeds 32 bits");
    if (!allowZero && v == 0u)
        throw std::invalid_argument(std::string(flag) + ": value must be non-zero");
    return static_cast<std::uint32_t>(v);
}

inline double parseDouble(std::string_view flag, const std::string& value)
{
    std::size_t used = 0u;
    double v = 0.0;
    try {
        v = std::stod(value, &used);
    } catch (const std::exception&) {
        used = std::string::npos;
    }
    if (used != value.size() || value.empty() || !std::isfinite(v))
        throw std::invalid_argument(std::string(flag) + ": expected a finite number, got '" + value + "'");
    return v;
}

inline void expectOneOf(std::string_view flag, const std::string& value, std::initializer_list<std::string_view> allowed)
{
    for (const auto a : allowed)
        if (value == a)
            return;
    std::string list;
    for (const auto a : allowed)
        list += (list.empty() ? "" : " or ") + std::string(a);
    throw std::invalid_argument(std::string(flag) + ": expected " + list + ", got '" + value + "'");
}

inline std::string lastError()
{
    char buf[512] = {0};
    gf_last_error(buf, sizeof(buf));
    return buf;
}

inline void cudaOrThrow(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

} // namespace gfcli
