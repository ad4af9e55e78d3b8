// antsRegistration-compatible front end for one SyN + CC stage on the synx C ABI.
//
// Same entry-point shape as the reference library call
// `int ants::antsRegistration(std::vector<std::string> args, std::ostream* out)`
// (Examples/include/antsRegistration.h:7-9): args are the command-line words without the
// program name; returns EXIT_SUCCESS / EXIT_FAILURE, exceptions never escape.
#pragma once

#include <ostream>
#include <string>
#include <vector>

namespace ants_b200 {

int antsRegistration(std::vector<std::string> args, std::ostream* out);

}  // namespace ants_b200

// The reference's own library symbol, `ants::antsRegistration` (Examples/include/antsRegistration.h:7-9,
// body Examples/antsRegistration.cxx:554-777), declared in include/antsRegistration.h, so that a
// wrapper compiled against the reference's header links against libantsRegistration_b200.so
// unchanged.  Forwards to ants_b200::antsRegistration.
#include "antsRegistration.h"
