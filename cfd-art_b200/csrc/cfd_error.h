// Error reporting shared by the library's translation units: records the
// message that cfd_last_error() returns on the calling thread and returns code.
#pragma once

int cfd_fail(int code, const char* fmt, ...);
