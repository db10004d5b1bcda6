// No C++ exception may cross the C ABI, nor leave a host worker thread (both
// would terminate the calling process).  guard_call runs a body and turns a
// host allocation failure into CULS_E_OOM and any other exception into
// CULS_E_INVALID, with a message for culs_last_error when `err` is given.
#pragma once
#include <exception>
#include <new>
#include <string>

#include "culs_b200.h"

namespace culs {

inline void note_error(std::string *err, const char *what) noexcept {
    if (!err) return;
    try {
        *err = what;
    } catch (...) {
    }
}

template <class F>
auto guard_call(std::string *err, F &&f) noexcept -> decltype(f()) {
    using R = decltype(f());
    try {
        return f();
    } catch (const std::bad_alloc &) {
        note_error(err, "host allocation failed");
        return (R)CULS_E_OOM;
    } catch (const std::exception &e) {
        note_error(err, e.what());
        return (R)CULS_E_INVALID;
    } catch (...) {
        note_error(err, "unexpected host exception");
        return (R)CULS_E_INVALID;
    }
}

}  // namespace culs
