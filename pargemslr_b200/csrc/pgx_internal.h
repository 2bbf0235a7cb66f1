// Library-internal helpers shared by the host-side translation units.
#pragma once

namespace pgx {

// Records msg as the calling thread's pgx_last_error() and returns code.
int set_error(int code, const char* msg);

}  // namespace pgx
