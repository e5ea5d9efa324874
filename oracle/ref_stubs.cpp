// Test infrastructure (the oracle), not product code.
//
// Link stubs for the reference's file-IO and glass-catalog functions. Their sources need the
// nlohmann/json library, which is not part of the reference tree, and the oracle never calls
// them: it builds SystemBatchHost directly from arrays. Any call reports that clearly.

#include "mikroptim/glass/catalog.hpp"
#include "mikroptim/io/system_json.hpp"

#include <stdexcept>

namespace mko {

namespace {
[[noreturn]] void unavailable(const char* what) {
    throw std::logic_error(std::string(what) + ": file IO and glass catalogs are not part of "
                                               "the oracle build");
}
} // namespace

bool Glass::in_range(double) const { unavailable("Glass::in_range"); }
double Glass::index(double) const { unavailable("Glass::index"); }
GlassCatalog GlassCatalog::from_file(const std::filesystem::path&) {
    unavailable("GlassCatalog::from_file");
}
void GlassCatalog::merge(const GlassCatalog&) { unavailable("GlassCatalog::merge"); }
const Glass* GlassCatalog::find(std::string_view) const { unavailable("GlassCatalog::find"); }
const Glass& GlassCatalog::at(std::string_view) const { unavailable("GlassCatalog::at"); }
SystemDescription read_system_file(const std::filesystem::path&, std::vector<std::string>*) {
    unavailable("read_system_file");
}
std::vector<std::filesystem::path> resolve_glass_catalogs(const SystemDescription&,
                                                          const std::filesystem::path&) {
    unavailable("resolve_glass_catalogs");
}

} // namespace mko
