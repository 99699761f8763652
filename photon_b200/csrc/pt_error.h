// The library's error type: thrown inside the library and turned into status codes at the C boundary.
// Free of CUDA so that host-only sources (the scene generator) compile without the toolkit.
#pragma once

#include <cstdint>
#include <string>

namespace ptw {

struct Error {
    int32_t code;  // a PT_ERR_* status
    std::string message;
};

}  // namespace ptw
