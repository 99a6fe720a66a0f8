// error.hpp -- per-thread last-error message behind mcg_last_error().
#pragma once
#include <string>

#include "mcg.h"

namespace mcg {

std::string &last_error();

inline void clear_error() { last_error().clear(); }

inline mcg_status fail(mcg_status code, const std::string &msg) {
    last_error() = msg;
    return code;
}

}  // namespace mcg
