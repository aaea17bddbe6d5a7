// Error state shared by every C entry point.
#include "common.cuh"

#include <string>

namespace rexlib_b200
{

namespace
{
thread_local std::string last_error_message;
}

const char *last_error_text() { return last_error_message.c_str(); }

void set_last_error(const std::string &message) { last_error_message = message; }

} // namespace rexlib_b200

extern "C" const char *rexlib_b200_last_error(void)
{
	return rexlib_b200::last_error_text();
}
