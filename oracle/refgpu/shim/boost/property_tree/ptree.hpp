// Stand-in for boost::property_tree::ptree: the reference's JSON scene
// loader names it, and the grid step driven through the C++ API never calls
// it; every accessor throws.
#pragma once
#include <stdexcept>
#include <string>
#include <utility>
namespace boost { namespace property_tree {
class ptree {
 public:
  typedef std::pair<const std::string, ptree> value_type;
  const ptree& get_child(const std::string&) const { throw std::runtime_error("ptree: JSON configuration is not supported"); }
  template <class T> T get_value() const { throw std::runtime_error("ptree: JSON configuration is not supported"); }
  const value_type* begin() const { return nullptr; }
  const value_type* end() const { return nullptr; }
};
} }
