// ref_enums.h -- this library's integer method codes (include/dream_sir.h:
// DREAM_FOC_*, DREAM_STEER_*, DREAM_APOD_*; include/dream_das.h:
// DREAM_ERR_LEVEL_*) mapped onto the reference's enum classes
// (include/dream.h). TEST INFRASTRUCTURE ONLY: shared by the drivers that call
// the reference's own code built by oracle/build_ref.sh.
#pragma once

#include "dream.h"

namespace ref_codes {

inline FocusMet foc_of(int m) {
  switch (m) {
    case 1: return FocusMet::x;
    case 2: return FocusMet::y;
    case 3: return FocusMet::xy;
    case 4: return FocusMet::x_y;
    case 5: return FocusMet::ud;
    default: return FocusMet::none;
  }
}

inline SteerMet steer_of(int m) {
  switch (m) {
    case 1: return SteerMet::x;
    case 2: return SteerMet::y;
    case 3: return SteerMet::xy;
    default: return SteerMet::none;
  }
}

// code 0 ("off") is not an ApodMet: the caller passes do_apod = false
inline ApodMet apod_of(int m) {
  switch (m) {
    case 1: return ApodMet::triangle;
    case 2: return ApodMet::gauss;
    case 3: return ApodMet::raised_cosine;
    case 4: return ApodMet::hann;
    case 5: return ApodMet::hamming;
    case 6: return ApodMet::simply_supported;
    case 7: return ApodMet::clamped;
    default: return ApodMet::ud;
  }
}

inline ErrorLevel err_of(int e) {
  switch (e) {
    case 1: return ErrorLevel::ignore;
    case 2: return ErrorLevel::warn;
    case 3: return ErrorLevel::stop;
    case 4: return ErrorLevel::parallel_stop;
    default: return ErrorLevel::none;
  }
}

}  // namespace ref_codes
