// gls_logging.h — TEST INFRASTRUCTURE ONLY. Stand-in for GlassImage's
// logging macros: every LOG_* stream discards what it is given.
#pragma once

#include <ostream>

namespace gls_shim {
inline std::ostream& null_log() {
    static std::ostream sink(nullptr);
    return sink;
}
}  // namespace gls_shim

#define LOG_INFO(tag) ::gls_shim::null_log()
#define LOG_DEBUG(tag) ::gls_shim::null_log()
#define LOG_WARNING(tag) ::gls_shim::null_log()
#define LOG_ERROR(tag) ::gls_shim::null_log()
