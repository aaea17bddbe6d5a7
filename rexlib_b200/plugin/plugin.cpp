// The rexlib plugin of the B200 backend: REXLIB_DEFINE_PLUGIN
// (include/rexlib/core/plugin_definition.hpp:26-50) defines the two C entry
// points rexlib's plugin loader looks up; register_at
// (include/rexlib/core/plugin.hpp:53) adds the "b200" device backend to the
// device service and this backend's program builders to the program
// service, after which execute() and the eager dispatcher reach the B200
// kernels through the unchanged operation declarations.
//
// The constructor checks that librexlib_b200.so, which holds the kernels,
// has the ABI these sources were compiled against; a mismatch throws, and
// rexlib_get_plugin then returns null, so rexlib skips the plugin.
#include "hardware.hpp"
#include "registry.hpp"

#include <rexlib_b200.h>

#include <rexlib/core/dispatch/program_service.hpp>
#include <rexlib/core/hardware/device_service.hpp>
#include <rexlib/core/plugin.hpp>
#include <rexlib/core/plugin_definition.hpp>
#include <rexlib/core/service_catalog.hpp>
#include <rexlib/core/version.hpp>

#include <memory>
#include <stdexcept>
#include <string>

// The ABI of the kernel library this plugin calls; a build can name another
// to stand for a plugin built against a different kernel library.
#ifndef REXLIB_B200_PLUGIN_KERNEL_ABI
#define REXLIB_B200_PLUGIN_KERNEL_ABI REXLIB_B200_ABI_VERSION
#endif

namespace rexlib_b200
{
namespace plugin
{

rexlib::program_builder_registry &get_program_builder_registry() noexcept
{
	static rexlib::program_builder_registry registry;
	return registry;
}

class b200_plugin final : public rexlib::plugin
{
public:
	b200_plugin()
	{
		const int32_t found = rexlib_b200_abi_version();
		if (found != REXLIB_B200_PLUGIN_KERNEL_ABI)
			throw std::runtime_error("rexlib_b200: the kernel library has ABI " + std::to_string(found) +
				", this plugin needs " + std::to_string(REXLIB_B200_PLUGIN_KERNEL_ABI));
	}

	const std::string &get_name() const noexcept override
	{
		static const std::string name("rexlib-b200");
		return name;
	}

	rexlib::version get_version() const noexcept override { return rexlib::version(0, 2, 0); }

	void register_at(rexlib::service_catalog &catalog) const override
	{
		catalog.get_service<rexlib::device_service>()->register_backend(std::make_unique<device_backend>());
		get_program_builder_registry().register_all(*catalog.get_service<rexlib::program_service>());
	}
};

} // namespace plugin
} // namespace rexlib_b200

REXLIB_DEFINE_PLUGIN(rexlib_b200::plugin::b200_plugin);
