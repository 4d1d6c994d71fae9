// abi_util.h -- error plumbing shared by the C-ABI entry points: every entry
// point runs its body inside guarded(), which turns a thrown Failure (or any
// std::exception) into a status code and a per-thread message, so nothing
// propagates across the extern "C" boundary and the host process is never
// aborted by the library.
#pragma once

#include <exception>
#include <memory>
#include <stdexcept>
#include <string>

#include "dgswem_cuda.h"

namespace dgswem {

struct Failure : std::runtime_error {
  int code;
  Failure(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

void set_last_error(const std::string& msg);

// The next MET_FORCING block of an NWS = 1 fort.22 reader (deck.cpp): NP
// records into wsx2, wsy2, pr2 (input node order); throws Failure.
void met_read_block(dgswem_met_reader* r, double* wsx2, double* wsy2, double* pr2);

template <typename F>
int guarded(F&& body) {
  try {
    body();
    return DGSWEM_OK;
  } catch (const Failure& f) {
    set_last_error(f.what());
    return f.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return DGSWEM_ERR_ARG;
  } catch (...) {
    set_last_error("unknown failure");
    return DGSWEM_ERR_ARG;
  }
}

}  // namespace dgswem
