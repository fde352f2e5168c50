// Minimal JSON reader for the drop-in FLOW driver: objects, arrays, strings,
// numbers, true/false/null.  Query helpers follow the conventions the
// reference's validators rely on (nlohmann::json 2.1.1 as used in
// src/InputOutput/JsonInput/**): size() of a missing value is 0, of a
// primitive 1, of an array/object its element count; count(key) is 0 or 1.
#pragma once
#include <cctype>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace jl {

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Value> arr;
    std::map<std::string, Value> obj;

    size_t size() const {
        switch (kind) {
            case Null: return 0;
            case Array: return arr.size();
            case Object: return obj.size();
            default: return 1;
        }
    }
    size_t count(const std::string& k) const { return kind == Object ? obj.count(k) : 0; }
    const Value& operator[](const std::string& k) const {
        static const Value none;
        if (kind != Object) return none;
        auto it = obj.find(k);
        return it == obj.end() ? none : it->second;
    }
    bool is_string(const char* s) const { return kind == String && str == s; }
};

class Parser {
public:
    explicit Parser(const std::string& text) : t_(text) {}
    Value parse() {
        Value v = value();
        ws();
        if (p_ != t_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string& t_;
    size_t p_ = 0;

    [[noreturn]] void fail(const std::string& why) {
        throw std::runtime_error("JSON parse error at offset " + std::to_string(p_) + ": " + why);
    }
    void ws() {
        while (p_ < t_.size() && std::isspace((unsigned char)t_[p_])) p_++;
    }
    bool eat(char c) {
        ws();
        if (p_ < t_.size() && t_[p_] == c) {
            p_++;
            return true;
        }
        return false;
    }
    void expect(char c) {
        if (!eat(c)) fail(std::string("expected '") + c + "'");
    }
    Value value() {
        ws();
        if (p_ >= t_.size()) fail("unexpected end");
        const char c = t_[p_];
        Value v;
        if (c == '{') {
            p_++;
            v.kind = Value::Object;
            if (eat('}')) return v;
            do {
                ws();
                Value k = string_value();
                expect(':');
                v.obj[k.str] = value();
            } while (eat(','));
            expect('}');
        } else if (c == '[') {
            p_++;
            v.kind = Value::Array;
            if (eat(']')) return v;
            do v.arr.push_back(value());
            while (eat(','));
            expect(']');
        } else if (c == '"') {
            v = string_value();
        } else if (t_.compare(p_, 4, "true") == 0) {
            p_ += 4;
            v.kind = Value::Bool;
            v.b = true;
        } else if (t_.compare(p_, 5, "false") == 0) {
            p_ += 5;
            v.kind = Value::Bool;
        } else if (t_.compare(p_, 4, "null") == 0) {
            p_ += 4;
        } else {
            const char* start = t_.c_str() + p_;
            char* end = nullptr;
            v.num = std::strtod(start, &end);
            if (end == start) fail("bad value");
            p_ += size_t(end - start);
            v.kind = Value::Number;
        }
        return v;
    }
    Value string_value() {
        if (p_ >= t_.size() || t_[p_] != '"') fail("expected string");
        p_++;
        Value v;
        v.kind = Value::String;
        while (p_ < t_.size() && t_[p_] != '"') {
            char c = t_[p_++];
            if (c == '\\' && p_ < t_.size()) {
                char e = t_[p_++];
                switch (e) {
                    case 'n': c = '\n'; break;
                    case 't': c = '\t'; break;
                    case 'r': c = '\r'; break;
                    case 'b': c = '\b'; break;
                    case 'f': c = '\f'; break;
                    case 'u':
                        if (p_ + 4 > t_.size()) fail("bad escape");
                        c = char(std::strtol(t_.substr(p_, 4).c_str(), nullptr, 16) & 0x7f);
                        p_ += 4;
                        break;
                    default: c = e;
                }
            }
            v.str.push_back(c);
        }
        if (p_ >= t_.size()) fail("unterminated string");
        p_++;
        return v;
    }
};

}  // namespace jl
