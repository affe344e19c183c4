// Drop-in for the reference header include/ftlm/version.hpp.
#pragma once

namespace ftlm {

const char* version_string();

}  // namespace ftlm
