// Minimal JSON reader for the three case files (setup.json, mesh.json,
// windturbine.json).  Numbers are converted with strtod, which rounds
// correctly, so a value reads back as the same double the reference's
// parser produces.  Only what the case files use is supported: objects,
// arrays, numbers, strings, true/false/null.
#pragma once

#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace dalm {

class Json {
public:
    enum Kind { Null, Bool, Number, String, Array, Object };

    Kind kind = Null;
    bool b = false;
    double num = 0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    static Json parse(const std::string &text) {
        size_t pos = 0;
        Json v = parse_value(text, pos);
        skip_ws(text, pos);
        if (pos != text.size()) fail(text, pos, "trailing characters");
        return v;
    }

    bool is_number() const { return kind == Number; }
    bool is_object() const { return kind == Object; }
    bool is_array() const { return kind == Array; }
    bool is_string() const { return kind == String; }

    bool contains(const std::string &key) const {
        if (kind != Object) return false;
        for (auto &kv : obj)
            if (kv.first == key) return true;
        return false;
    }
    const Json &operator[](const std::string &key) const {
        if (kind != Object) throw std::runtime_error("JSON: not an object when reading \"" + key + "\"");
        for (auto &kv : obj)
            if (kv.first == key) return kv.second;
        throw std::runtime_error("JSON: missing key \"" + key + "\"");
    }
    const Json &operator[](size_t i) const {
        if (kind != Array) throw std::runtime_error("JSON: not an array");
        if (i >= arr.size()) throw std::runtime_error("JSON: index out of range");
        return arr[i];
    }
    size_t size() const { return kind == Array ? arr.size() : (kind == Object ? obj.size() : 0); }
    double number() const {
        if (kind != Number) throw std::runtime_error("JSON: expected a number");
        return num;
    }
    const std::string &string() const {
        if (kind != String) throw std::runtime_error("JSON: expected a string");
        return str;
    }
    std::vector<double> numbers() const {
        std::vector<double> out;
        for (size_t i = 0; i < size(); i++) out.push_back((*this)[i].number());
        return out;
    }

private:
    [[noreturn]] static void fail(const std::string &t, size_t pos, const char *what) {
        (void)t;
        throw std::runtime_error(std::string("JSON parse error at offset ") + std::to_string(pos) +
                                 ": " + what);
    }
    static void skip_ws(const std::string &t, size_t &pos) {
        while (pos < t.size() && (t[pos] == ' ' || t[pos] == '\n' || t[pos] == '\r' || t[pos] == '\t'))
            pos++;
    }
    static Json parse_value(const std::string &t, size_t &pos) {
        skip_ws(t, pos);
        if (pos >= t.size()) fail(t, pos, "unexpected end");
        char c = t[pos];
        Json v;
        if (c == '{') {
            v.kind = Object;
            pos++;
            skip_ws(t, pos);
            if (pos < t.size() && t[pos] == '}') { pos++; return v; }
            while (true) {
                skip_ws(t, pos);
                Json key = parse_value(t, pos);
                if (key.kind != String) fail(t, pos, "object key must be a string");
                skip_ws(t, pos);
                if (pos >= t.size() || t[pos] != ':') fail(t, pos, "expected ':'");
                pos++;
                Json val = parse_value(t, pos);
                v.obj.emplace_back(key.str, std::move(val));
                skip_ws(t, pos);
                if (pos < t.size() && t[pos] == ',') { pos++; continue; }
                if (pos < t.size() && t[pos] == '}') { pos++; break; }
                fail(t, pos, "expected ',' or '}'");
            }
        } else if (c == '[') {
            v.kind = Array;
            pos++;
            skip_ws(t, pos);
            if (pos < t.size() && t[pos] == ']') { pos++; return v; }
            while (true) {
                v.arr.push_back(parse_value(t, pos));
                skip_ws(t, pos);
                if (pos < t.size() && t[pos] == ',') { pos++; continue; }
                if (pos < t.size() && t[pos] == ']') { pos++; break; }
                fail(t, pos, "expected ',' or ']'");
            }
        } else if (c == '"') {
            v.kind = String;
            pos++;
            while (pos < t.size() && t[pos] != '"') {
                if (t[pos] == '\\' && pos + 1 < t.size()) {
                    char e = t[pos + 1];
                    v.str += (e == 'n') ? '\n' : (e == 't') ? '\t' : e;
                    pos += 2;
                } else {
                    v.str += t[pos++];
                }
            }
            if (pos >= t.size()) fail(t, pos, "unterminated string");
            pos++;
        } else if (t.compare(pos, 4, "true") == 0) {
            v.kind = Bool; v.b = true; pos += 4;
        } else if (t.compare(pos, 5, "false") == 0) {
            v.kind = Bool; v.b = false; pos += 5;
        } else if (t.compare(pos, 4, "null") == 0) {
            v.kind = Null; pos += 4;
        } else {
            const char *start = t.c_str() + pos;
            char *end = nullptr;
            double d = std::strtod(start, &end);
            if (end == start) fail(t, pos, "invalid value");
            v.kind = Number;
            v.num = d;
            pos += (size_t)(end - start);
        }
        return v;
    }
};

}  // namespace dalm
