// The registry the B200 backend's program builders add themselves to during
// static initialization (the pattern of
// include/rexlib/core/dispatch/program_builder_registration.hpp:26); the
// plugin registers them all at the program service when rexlib loads it.
#pragma once

#include <rexlib/core/dispatch/program_builder_registry.hpp>

namespace rexlib_b200
{
namespace plugin
{

rexlib::program_builder_registry &get_program_builder_registry() noexcept;

} // namespace plugin
} // namespace rexlib_b200
