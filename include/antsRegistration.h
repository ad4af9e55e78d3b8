/* C++ library entry of the antsRegistration SyN + CC stage, for wrappers that bind the reference's
 * library call.
 *
 * Replaces `int ants::antsRegistration(std::vector<std::string>, std::ostream*)`
 * (Examples/include/antsRegistration.h:7-9; body Examples/antsRegistration.cxx:554-777) with the
 * same namespace, name, argument meaning and return convention: `args` are the command-line words
 * without the program name, the result is EXIT_SUCCESS or EXIT_FAILURE, and no exception escapes.
 * `out_stream` receives the verbose log (std::cout when NULL).  Exported by
 * ants_b200/libantsRegistration_b200.so, which runs the stage on the GPU through the C ABI of
 * synx.h.  The options it accepts are those of one SyN + CC stage; others fail with EXIT_FAILURE
 * and a message on stderr. */
#ifndef SYNX_ANTSREGISTRATION_H
#define SYNX_ANTSREGISTRATION_H

#include <ostream>
#include <string>
#include <vector>

namespace ants {
extern int antsRegistration(std::vector<std::string> args, std::ostream* out_stream);
}  // namespace ants

#endif /* SYNX_ANTSREGISTRATION_H */
