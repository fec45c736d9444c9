#pragma once
// Version of the limbforge API these headers provide (the reference's include/limbforge/version.hpp
// interface): the 1.3 API, so that callers' version checks pass unchanged.  library_version() asks the
// loaded liblimbforge_b200.so which API version it implements.
#define LIMBFORGE_VERSION_MAJOR 1
#define LIMBFORGE_VERSION_MINOR 3
#define LIMBFORGE_VERSION_PATCH 1
#define LIMBFORGE_API_VERSION LIMBFORGE_VERSION_MAJOR
#define LIMBFORGE_DETAIL_STRINGIFY_IMPL(x) #x
#define LIMBFORGE_DETAIL_STRINGIFY(x) LIMBFORGE_DETAIL_STRINGIFY_IMPL(x)
#define LIMBFORGE_VERSION_STRING \
    LIMBFORGE_DETAIL_STRINGIFY(LIMBFORGE_VERSION_MAJOR) "." LIMBFORGE_DETAIL_STRINGIFY(LIMBFORGE_VERSION_MINOR) "." \
    LIMBFORGE_DETAIL_STRINGIFY(LIMBFORGE_VERSION_PATCH)
#define LIMBFORGE_VERSION_AT_LEAST(major, minor, patch)                                                        \
    (LIMBFORGE_VERSION_MAJOR > (major) ||                                                                      \
     (LIMBFORGE_VERSION_MAJOR == (major) &&                                                                    \
      (LIMBFORGE_VERSION_MINOR > (minor) || (LIMBFORGE_VERSION_MINOR == (minor) && LIMBFORGE_VERSION_PATCH >= (patch)))))

#include <stdexcept>
#include <string>
#include "../limbforge_b200.h"

namespace limbforge {
struct Version { unsigned major, minor, patch; };
inline constexpr Version header_version{LIMBFORGE_VERSION_MAJOR, LIMBFORGE_VERSION_MINOR, LIMBFORGE_VERSION_PATCH};
inline constexpr unsigned api_version = LIMBFORGE_API_VERSION;
constexpr bool version_at_least(Version available, Version required) noexcept {
    return available.major != required.major ? available.major > required.major
         : available.minor != required.minor ? available.minor > required.minor
         : available.patch >= required.patch;
}
// Same major, and at least the required release.
constexpr bool version_compatible(Version available, Version required) noexcept {
    return available.major == required.major && version_at_least(available, required);
}
inline Version library_version() noexcept {
    Version v{0, 0, 0};
    lf_api_version(&v.major, &v.minor, &v.patch);
    return v;
}
inline const char* library_version_string() noexcept { return lf_version(); }
// std::runtime_error when the loaded library's major differs or it is older than `required` (any difference with exact).
inline void require_library_version(Version required, bool exact = false) {
    const Version v = library_version();
    const bool good = exact ? (v.major == required.major && v.minor == required.minor && v.patch == required.patch) : version_compatible(v, required);
    if (!good)
        throw std::runtime_error("limbforge library " + std::to_string(v.major) + "." + std::to_string(v.minor) + "." + std::to_string(v.patch) +
                                 " does not satisfy " + std::to_string(required.major) + "." + std::to_string(required.minor) + "." +
                                 std::to_string(required.patch));
}
inline void check_library_version() { require_library_version(header_version, true); }
}  // namespace limbforge
