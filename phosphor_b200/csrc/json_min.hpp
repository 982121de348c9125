// json_min.hpp — a small JSON reader for the glTF scene loader: objects, arrays, strings (with
// \uXXXX escapes encoded as UTF-8), numbers, true/false/null.  Parses a whole document into a
// tree of Json values; errors throw std::runtime_error with the byte offset.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace phx {

struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::map<std::string, Json> obj;

    bool has(const std::string &k) const { return kind == Object && obj.count(k) != 0; }
    const Json &operator[](const std::string &k) const {
        static const Json null_value;
        if (kind != Object)
            return null_value;
        auto it = obj.find(k);
        return it == obj.end() ? null_value : it->second;
    }
    const Json &operator[](size_t i) const {
        static const Json null_value;
        return (kind == Array && i < arr.size()) ? arr[i] : null_value;
    }
    size_t size() const { return kind == Array ? arr.size() : kind == Object ? obj.size() : 0; }
    double number(double dflt) const { return kind == Number ? num : dflt; }
    int64_t integer(int64_t dflt) const { return kind == Number ? (int64_t)num : dflt; }
    std::string string(const std::string &dflt = "") const { return kind == String ? str : dflt; }
};

class JsonParser {
  public:
    explicit JsonParser(const std::string &text) : s_(text) {}
    Json parse() {
        Json v = value();
        ws();
        if (i_ != s_.size())
            fail("trailing characters");
        return v;
    }

  private:
    const std::string &s_;
    size_t i_ = 0;
    int depth_ = 0;

    [[noreturn]] void fail(const char *what) const {
        throw std::runtime_error(std::string("JSON: ") + what + " at byte " + std::to_string(i_));
    }
    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\n' || s_[i_] == '\r' || s_[i_] == '\t'))
            i_++;
    }
    bool lit(const char *w) {
        size_t n = std::char_traits<char>::length(w);
        if (s_.compare(i_, n, w) == 0) {
            i_ += n;
            return true;
        }
        return false;
    }
    Json value() {
        ws();
        if (i_ >= s_.size())
            fail("unexpected end");
        if (++depth_ > 256)
            fail("nesting too deep");
        Json v;
        const char c = s_[i_];
        if (c == '{') {
            v.kind = Json::Object;
            i_++;
            ws();
            if (i_ < s_.size() && s_[i_] == '}') {
                i_++;
            } else {
                for (;;) {
                    ws();
                    if (i_ >= s_.size() || s_[i_] != '"')
                        fail("expected a key");
                    std::string k = string_body();
                    ws();
                    if (i_ >= s_.size() || s_[i_] != ':')
                        fail("expected ':'");
                    i_++;
                    v.obj[k] = value();
                    ws();
                    if (i_ < s_.size() && s_[i_] == ',') {
                        i_++;
                        continue;
                    }
                    if (i_ < s_.size() && s_[i_] == '}') {
                        i_++;
                        break;
                    }
                    fail("expected ',' or '}'");
                }
            }
        } else if (c == '[') {
            v.kind = Json::Array;
            i_++;
            ws();
            if (i_ < s_.size() && s_[i_] == ']') {
                i_++;
            } else {
                for (;;) {
                    v.arr.push_back(value());
                    ws();
                    if (i_ < s_.size() && s_[i_] == ',') {
                        i_++;
                        continue;
                    }
                    if (i_ < s_.size() && s_[i_] == ']') {
                        i_++;
                        break;
                    }
                    fail("expected ',' or ']'");
                }
            }
        } else if (c == '"') {
            v.kind = Json::String;
            v.str = string_body();
        } else if (lit("true")) {
            v.kind = Json::Bool;
            v.b = true;
        } else if (lit("false")) {
            v.kind = Json::Bool;
        } else if (lit("null")) {
            v.kind = Json::Null;
        } else if (c == '-' || (c >= '0' && c <= '9')) {
            v.kind = Json::Number;
            const char *start = s_.c_str() + i_;
            char *end = nullptr;
            v.num = std::strtod(start, &end);
            if (end == start)
                fail("bad number");
            i_ += (size_t)(end - start);
        } else {
            fail("unexpected character");
        }
        depth_--;
        return v;
    }
    static void utf8(std::string &out, uint32_t cp) {
        if (cp < 0x80) {
            out += (char)cp;
        } else if (cp < 0x800) {
            out += (char)(0xC0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18));
            out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (i_ + 4 > s_.size())
            fail("bad \\u escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; k++) {
            char h = s_[i_++];
            v <<= 4;
            if (h >= '0' && h <= '9')
                v |= (uint32_t)(h - '0');
            else if (h >= 'a' && h <= 'f')
                v |= (uint32_t)(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F')
                v |= (uint32_t)(h - 'A' + 10);
            else
                fail("bad \\u escape");
        }
        return v;
    }
    std::string string_body() {
        i_++; // opening quote
        std::string out;
        while (i_ < s_.size()) {
            char c = s_[i_++];
            if (c == '"')
                return out;
            if (c != '\\') {
                out += c;
                continue;
            }
            if (i_ >= s_.size())
                break;
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
                uint32_t cp = hex4();
                if (cp >= 0xD800 && cp < 0xDC00 && i_ + 6 <= s_.size() && s_[i_] == '\\' && s_[i_ + 1] == 'u') {
                    i_ += 2;
                    uint32_t lo = hex4();
                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                }
                utf8(out, cp);
                break;
            }
            default:
                fail("bad escape");
            }
        }
        fail("unterminated string");
    }
};

} // namespace phx
