// Minimal JSON reader for the detector configuration objects.
//
// The reference parses its config with nlohmann::json (a git submodule) and
// reads flat objects of numbers, booleans and strings
// (cpp/lib/apsm/apsm_noma_detector.cu:348-383).  This reader covers full JSON
// syntax (nested objects/arrays are parsed and kept as raw values) so that any
// document the reference accepts parses here too; only the value kinds the
// factory reads are exposed.
#pragma once

#include <cctype>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace apsm {

struct JsonValue {
    enum Kind { Null, Bool, Number, String, Object, Array } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<std::pair<std::string, JsonValue>> members; // Object, insertion order
    std::vector<JsonValue> items;                           // Array

    const JsonValue* find(const std::string& key) const
    {
        for (const auto& m : members)
            if (m.first == key) return &m.second;
        return nullptr;
    }
};

class JsonParser {
public:
    explicit JsonParser(const std::string& text) : s_(text), i_(0) {}

    JsonValue parse()
    {
        JsonValue v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string& s_;
    size_t i_;

    [[noreturn]] void fail(const char* what) const
    {
        throw std::invalid_argument(std::string("JSON parse error at offset ") + std::to_string(i_) + ": " + what);
    }
    void ws()
    {
        while (i_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[i_]))) ++i_;
    }
    bool lit(const char* w)
    {
        size_t n = std::char_traits<char>::length(w);
        if (s_.compare(i_, n, w) == 0) {
            i_ += n;
            return true;
        }
        return false;
    }
    JsonValue value()
    {
        ws();
        if (i_ >= s_.size()) fail("unexpected end");
        char c = s_[i_];
        JsonValue v;
        if (c == '{') {
            v.kind = JsonValue::Object;
            ++i_;
            ws();
            if (i_ < s_.size() && s_[i_] == '}') { ++i_; return v; }
            for (;;) {
                ws();
                if (i_ >= s_.size() || s_[i_] != '"') fail("expected key");
                std::string k = string();
                ws();
                if (i_ >= s_.size() || s_[i_] != ':') fail("expected ':'");
                ++i_;
                JsonValue m = value();
                bool replaced = false;
                for (auto& e : v.members)
                    if (e.first == k) { e.second = m; replaced = true; }
                if (!replaced) v.members.emplace_back(k, m);
                ws();
                if (i_ < s_.size() && s_[i_] == ',') { ++i_; continue; }
                if (i_ < s_.size() && s_[i_] == '}') { ++i_; return v; }
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = JsonValue::Array;
            ++i_;
            ws();
            if (i_ < s_.size() && s_[i_] == ']') { ++i_; return v; }
            for (;;) {
                v.items.push_back(value());
                ws();
                if (i_ < s_.size() && s_[i_] == ',') { ++i_; continue; }
                if (i_ < s_.size() && s_[i_] == ']') { ++i_; return v; }
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = JsonValue::String;
            v.str = string();
            return v;
        }
        if (lit("true")) { v.kind = JsonValue::Bool; v.b = true; return v; }
        if (lit("false")) { v.kind = JsonValue::Bool; v.b = false; return v; }
        if (lit("null")) { v.kind = JsonValue::Null; return v; }
        if (c == '-' || (c >= '0' && c <= '9')) {
            const char* begin = s_.c_str() + i_;
            char* end = nullptr;
            v.kind = JsonValue::Number;
            v.num = std::strtod(begin, &end);
            if (end == begin) fail("bad number");
            i_ += size_t(end - begin);
            return v;
        }
        fail("unexpected character");
    }
    std::string string()
    {
        std::string out;
        ++i_; // opening quote
        while (i_ < s_.size()) {
            char c = s_[i_++];
            if (c == '"') return out;
            if (c == '\\') {
                if (i_ >= s_.size()) break;
                char e = s_[i_++];
                switch (e) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    if (i_ + 4 > s_.size()) fail("bad \\u escape");
                    unsigned cp = unsigned(std::strtoul(s_.substr(i_, 4).c_str(), nullptr, 16));
                    i_ += 4;
                    if (cp < 0x80) out += char(cp);
                    else if (cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F)); }
                    else { out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F)); }
                    break;
                }
                default: fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        fail("unterminated string");
    }
};

inline JsonValue parse_json(const std::string& text) { return JsonParser(text).parse(); }

} // namespace apsm
