// error.cpp -- per-thread last-error storage.
#include "error.hpp"

namespace mcg {

std::string &last_error() {
    thread_local std::string msg;
    return msg;
}

}  // namespace mcg

extern "C" const char *mcg_last_error(void) { return mcg::last_error().c_str(); }
