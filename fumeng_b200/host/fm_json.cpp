#include "fm_json.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace fmhost {

namespace {

struct Parser {
    const char* p;
    const char* end;

    [[noreturn]] void fail(const char* what)
    {
        throw std::runtime_error(std::string("JSON parse error: ") + what);
    }
    void ws()
    {
        while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    }
    bool lit(const char* s)
    {
        const size_t n = std::strlen(s);
        if ((size_t)(end - p) >= n && std::strncmp(p, s, n) == 0) {
            p += n;
            return true;
        }
        return false;
    }
    std::string string_value()
    {
        if (*p != '"') fail("expected string");
        ++p;
        std::string out;
        while (p < end && *p != '"') {
            if (*p == '\\') {
                ++p;
                if (p >= end) fail("bad escape");
                switch (*p) {
                case 'n': out += '\n'; break;
                case 't': out += '\t'; break;
                case 'r': out += '\r'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'u': {
                    if (end - p < 5) fail("bad unicode escape");
                    const unsigned cp = (unsigned)std::strtoul(std::string(p + 1, p + 5).c_str(), nullptr, 16);
                    if (cp < 0x80) {
                        out += (char)cp;
                    } else if (cp < 0x800) {
                        out += (char)(0xC0 | (cp >> 6));
                        out += (char)(0x80 | (cp & 0x3F));
                    } else {
                        out += (char)(0xE0 | (cp >> 12));
                        out += (char)(0x80 | ((cp >> 6) & 0x3F));
                        out += (char)(0x80 | (cp & 0x3F));
                    }
                    p += 4;
                    break;
                }
                default: out += *p;
                }
                ++p;
            } else {
                out += *p++;
            }
        }
        if (p >= end) fail("unterminated string");
        ++p;
        return out;
    }
    Json value()
    {
        ws();
        if (p >= end) fail("unexpected end");
        Json j;
        if (*p == '{') {
            ++p;
            j.kind = Json::Object;
            ws();
            if (*p == '}') {
                ++p;
                return j;
            }
            for (;;) {
                ws();
                std::string k = string_value();
                ws();
                if (*p != ':') fail("expected ':'");
                ++p;
                j.obj.emplace_back(std::move(k), value());
                ws();
                if (*p == ',') {
                    ++p;
                    continue;
                }
                if (*p == '}') {
                    ++p;
                    return j;
                }
                fail("expected ',' or '}'");
            }
        }
        if (*p == '[') {
            ++p;
            j.kind = Json::Array;
            ws();
            if (*p == ']') {
                ++p;
                return j;
            }
            for (;;) {
                j.arr.push_back(value());
                ws();
                if (*p == ',') {
                    ++p;
                    continue;
                }
                if (*p == ']') {
                    ++p;
                    return j;
                }
                fail("expected ',' or ']'");
            }
        }
        if (*p == '"') {
            j.kind = Json::String;
            j.str = string_value();
            return j;
        }
        if (lit("true")) {
            j.kind = Json::Bool;
            j.b = true;
            return j;
        }
        if (lit("false")) {
            j.kind = Json::Bool;
            return j;
        }
        if (lit("null")) return j;
        char* e = nullptr;
        j.num = std::strtod(p, &e);
        if (e == p) fail("bad value");
        j.kind = Json::Number;
        p = e;
        return j;
    }
};

void type_error(const char* name) { std::fprintf(stderr, "[fumeng_b200] Failed when parsing %s.\n", name); }

}  // namespace

bool Json::has(const std::string& k) const { return find(k) != nullptr; }

const Json* Json::find(const std::string& k) const
{
    if (kind != Object) return nullptr;
    for (const auto& kv : obj)
        if (kv.first == k) return &kv.second;
    return nullptr;
}

const Json& Json::at(const std::string& k) const
{
    const Json* j = find(k);
    if (!j) throw std::runtime_error("missing JSON field: " + k);
    return *j;
}

Json Json::parse(const std::string& text)
{
    Parser ps{text.data(), text.data() + text.size()};
    Json j = ps.value();
    ps.ws();
    if (ps.p != ps.end) ps.fail("trailing characters");
    return j;
}

void load(const Json& j, const char* name, double& v)
{
    const Json* f = j.find(name);
    if (!f) return;
    if (f->is_number())
        v = f->num;
    else
        type_error(name);
}
void load(const Json& j, const char* name, float& v)
{
    double d = v;
    const Json* f = j.find(name);
    if (!f) return;
    if (f->is_number()) {
        d = f->num;
        v = (float)d;
    } else {
        type_error(name);
    }
}
void load(const Json& j, const char* name, int& v)
{
    const Json* f = j.find(name);
    if (!f) return;
    if (f->is_number())
        v = (int)f->num;
    else
        type_error(name);
}
void load(const Json& j, const char* name, bool& v)
{
    const Json* f = j.find(name);
    if (!f) return;
    if (f->kind == Json::Bool)
        v = f->b;
    else
        type_error(name);
}
void load(const Json& j, const char* name, std::string& v)
{
    const Json* f = j.find(name);
    if (!f) return;
    if (f->is_string())
        v = f->str;
    else
        type_error(name);
}
void load_vec3(const Json& j, const char* name, float v[3])
{
    const Json* f = j.find(name);
    if (!f) return;
    if (!f->is_array()) {
        type_error(name);
        return;
    }
    std::vector<float> nums;
    for (const auto& e : f->arr) {
        if (!e.is_number()) {
            type_error(name);
            return;
        }
        nums.push_back((float)e.num);
    }
    if (nums.empty()) return;
    if (nums.size() < 3) {
        v[0] = v[1] = v[2] = nums[0];
        return;
    }
    v[0] = nums[0];
    v[1] = nums[1];
    v[2] = nums[2];
}

}  // namespace fmhost
