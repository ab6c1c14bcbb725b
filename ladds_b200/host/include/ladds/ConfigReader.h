// ConfigReader.h -- the YAML configuration of the hot path.
//
// Mirrors the access contract of the reference's ConfigReader
// (src/ladds/io/ConfigReader.h:23-230): values are addressed by '/'-separated
// paths, get<T>(path, fallback) returns the fallback for a missing key and
// writes it into the tree (so later reads agree), a missing key without a
// fallback throws std::runtime_error.  yaml-cpp is not available here, so the
// reader parses the block-mapping subset of YAML the LADDS configuration files
// use (nested "key: value" maps by indentation, '#' comments, plain or quoted
// scalars).
#pragma once
#include <map>
#include <memory>
#include <optional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace ladds {

class ConfigReader {
 public:
  struct Node {
    std::string value;  // scalar (empty for maps)
    std::map<std::string, std::unique_ptr<Node>> children;
  };

  ConfigReader();
  static ConfigReader fromFile(const std::string &path);
  static ConfigReader fromString(const std::string &yaml);

  template <class T>
  T get(const std::string &valuePath, std::optional<T> fallbackValue = std::nullopt) {
    const Node *n = find(valuePath);
    if (!n || !n->children.empty()) {
      if (!fallbackValue.has_value()) throw std::runtime_error("Config option not found: " + valuePath);
      setValue(valuePath, fallbackValue.value());
      parsed_[valuePath] = toString(fallbackValue.value());
      return fallbackValue.value();
    }
    parsed_[valuePath] = n->value;
    return fromString<T>(n->value, valuePath);
  }

  bool defines(const std::string &valuePath) const { return find(valuePath) != nullptr; }

  template <class T>
  void setValue(const std::string &valuePath, const T &value) {
    insert(valuePath)->value = toString(value);
  }

  // values read so far (path -> text), like printParsedValues()
  const std::map<std::string, std::string> &parsedValues() const { return parsed_; }
  std::string dump() const;

 private:
  const Node *find(const std::string &path) const;
  Node *insert(const std::string &path);
  static std::vector<std::string> split(const std::string &path);

  template <class T>
  static std::string toString(const T &v) {
    if constexpr (std::is_same_v<T, std::string>) {
      return v;
    } else if constexpr (std::is_same_v<T, bool>) {
      return v ? "true" : "false";
    } else if constexpr (std::is_convertible_v<T, const char *>) {
      return std::string(v);
    } else {
      std::ostringstream os;
      os.precision(17);
      os << v;
      return os.str();
    }
  }

  template <class T>
  static T fromString(const std::string &s, const std::string &path) {
    if constexpr (std::is_same_v<T, std::string>) {
      return s;
    } else if constexpr (std::is_same_v<T, bool>) {
      if (s == "true" || s == "True" || s == "TRUE" || s == "yes" || s == "on" || s == "1") return true;
      if (s == "false" || s == "False" || s == "FALSE" || s == "no" || s == "off" || s == "0") return false;
      throw std::runtime_error("Config option " + path + " is not a bool: " + s);
    } else {
      std::istringstream is(s);
      T v{};
      is >> v;
      if (is.fail()) throw std::runtime_error("Config option " + path + " has the wrong type: " + s);
      return v;
    }
  }

  std::unique_ptr<Node> root_;
  std::map<std::string, std::string> parsed_;
};

}  // namespace ladds
