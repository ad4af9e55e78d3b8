// antsApplyTransforms-compatible front end for displacement-field transforms on the synx C ABI.
//
// Same entry-point shape as the reference library call
// `int ants::antsApplyTransforms(std::vector<std::string> args, std::ostream* out)`
// (Examples/include/antsApplyTransforms.h): args are the command-line words without the program
// name; returns EXIT_SUCCESS / EXIT_FAILURE, exceptions never escape.
#pragma once

#include <ostream>
#include <string>
#include <vector>

namespace ants_b200 {

int antsApplyTransforms(std::vector<std::string> args, std::ostream* out);

}  // namespace ants_b200
