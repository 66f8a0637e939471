// Minimal JSON reader for the scene files (objects, arrays, numbers, strings, booleans,
// null).  Numbers are parsed with strtod, as the reference's JSON library reads them.
#pragma once
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace fmhost {

struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;   // insertion order kept

    bool is_object() const { return kind == Object; }
    bool is_array() const { return kind == Array; }
    bool is_number() const { return kind == Number; }
    bool is_string() const { return kind == String; }
    bool has(const std::string& k) const;
    const Json& at(const std::string& k) const;   // throws when missing
    const Json* find(const std::string& k) const;

    static Json parse(const std::string& text);
};

// Field loaders with the reference's rules (core/config.h:22-100): a missing field keeps
// the default; a vec3 given with fewer than 3 numbers broadcasts its first number; a
// field of the wrong type keeps the default and reports an error on stderr.
void load(const Json& j, const char* name, double& v);
void load(const Json& j, const char* name, float& v);
void load(const Json& j, const char* name, int& v);
void load(const Json& j, const char* name, bool& v);
void load(const Json& j, const char* name, std::string& v);
void load_vec3(const Json& j, const char* name, float v[3]);

}  // namespace fmhost
