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
