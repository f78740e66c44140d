// life_simulation_b200/csrc/abi_guard.h -- keeps C++ exceptions inside the
// library: every extern "C" entry point of include/lenia_b200.h runs its body
// through abi_guard, which turns an exception into a status code and a
// message (the reference's boundary throws nothing either: setup problems are
// printed and fallen back from, LeniaModule::setup, Lenia.cpp:245-313).
#pragma once

#include <exception>
#include <new>
#include <string>

#include "../../include/lenia_b200.h"

namespace lenia {

// Runs `body` (returning an int status). std::bad_alloc (a host allocation
// failed) becomes LENIA_ERR_CUDA like a failed device allocation; any other
// exception becomes LENIA_ERR_STATE. The message goes to *msg when msg is not
// null; storing it cannot throw out of here either.
template <typename F>
int abi_guard(std::string* msg, F&& body) noexcept {
    const auto note = [msg](const char* what) noexcept {
        if (!msg) return;
        try {
            *msg = what;
        } catch (...) {
        }
    };
    try {
        return body();
    } catch (const std::bad_alloc&) {
        note("host allocation failed");
        return LENIA_ERR_CUDA;
    } catch (const std::exception& e) {
        note(e.what());
        return LENIA_ERR_STATE;
    } catch (...) {
        note("unknown C++ exception");
        return LENIA_ERR_STATE;
    }
}

}  // namespace lenia
