/* C++ library entry of antsApplyTransforms for displacement-field and linear transform stacks, for
 * wrappers that bind the reference's library call.
 *
 * Replaces `int ants::antsApplyTransforms(std::vector<std::string>, std::ostream*)`
 * (Examples/include/antsApplyTransforms.h:4-10; body Examples/antsApplyTransforms.cxx:1279-) with the
 * same namespace, name, argument meaning and return convention: `args` are the command-line words
 * without the program name, the result is EXIT_SUCCESS or EXIT_FAILURE, and no exception escapes.
 * `out_stream` receives the verbose log (std::cout when NULL).  Exported by
 * ants_b200/libantsApplyTransforms_b200.so, which resamples on the GPU through the C ABI of synx.h.
 * The transforms it accepts are displacement fields, the linear types of synx_read_linear_transform
 * and text composites of them; others fail with EXIT_FAILURE and a message on stderr. */
#ifndef SYNX_ANTSAPPLYTRANSFORMS_H
#define SYNX_ANTSAPPLYTRANSFORMS_H

#include <ostream>
#include <string>
#include <vector>

namespace ants {
extern int antsApplyTransforms(std::vector<std::string> args, std::ostream* out_stream);
}  // namespace ants

#endif /* SYNX_ANTSAPPLYTRANSFORMS_H */
