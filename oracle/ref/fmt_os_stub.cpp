// Link stubs for the fmt file-output symbols the reference declares through <fmt/os.h> but whose
// definitions live in fmt's compiled library (not available here).  The reference only uses them to
// write error logs on a negative Jacobian (Mesh.cpp:505-513); parity runs use valid grids, so
// reaching any of them is reported and ends the run.  TEST INFRASTRUCTURE ONLY.
#include <cstdio>
#include <cstdlib>

#include "fmt/os.h"

namespace {
[[noreturn]] void unreachable_log(const char *what) {
  std::fprintf(stderr, "reference error-log path reached (%s); not supported in parity runs\n", what);
  std::abort();
}
}  // namespace

FMT_BEGIN_NAMESPACE
namespace detail {
file_buffer::file_buffer(cstring_view, const ostream_params &) { unreachable_log("fmt::output_file"); }
file_buffer::~file_buffer() {}
void file_buffer::grow(size_t) { unreachable_log("fmt::file_buffer::grow"); }
}  // namespace detail
void file::close() {}
size_t file::write(const void *, size_t) { unreachable_log("fmt::file::write"); }
file::~file() noexcept {}
ostream::~ostream() {}
FMT_END_NAMESPACE
