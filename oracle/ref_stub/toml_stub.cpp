// TOML front end stand-in for the reference harness: the harness fills the
// controller's command map directly and never parses an mdin file.
#include <map>
#include <string>

namespace sponge::toml_wrap
{
bool ParseAndFlatten(const std::string&, const std::string&, std::map<std::string, std::string>*,
                     std::string* error_message)
{
    if (error_message) *error_message = "TOML input is not available in the reference harness";
    return false;
}
}  // namespace sponge::toml_wrap
