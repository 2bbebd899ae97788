// Strict JSON reader for the hardware profile and design-space files given to
// Context::init.  Same contract as the reference's config parser
// (src/framework/json_config.hpp:14-135): a top-level object, no duplicate keys, no trailing
// text, integers that must not carry a fraction or exponent, errors thrown as
// std::runtime_error.  Implementation is independent.
#pragma once
#include <cerrno>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace bfly {
namespace json {

struct Node {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    std::string text;                  // number literal or string value
    std::vector<Node> items;           // Array
    std::map<std::string, Node> members;  // Object

    bool has(const std::string& key) const { return kind == Object && members.count(key) != 0; }
    const Node& get(const std::string& key) const {
        if (kind != Object) throw std::runtime_error("expected an object holding '" + key + "'");
        auto it = members.find(key);
        if (it == members.end()) throw std::runtime_error("missing field '" + key + "'");
        return it->second;
    }
    long long asInt() const {
        if (kind != Number || text.find_first_of(".eE") != std::string::npos)
            throw std::runtime_error("expected an integer, got '" + text + "'");
        errno = 0;
        char* end = nullptr;
        long long v = std::strtoll(text.c_str(), &end, 10);
        if (errno || !end || *end) throw std::runtime_error("integer out of range: " + text);
        return v;
    }
    double asDouble() const {
        if (kind != Number) throw std::runtime_error("expected a number");
        return std::strtod(text.c_str(), nullptr);
    }
    const std::string& asString() const {
        if (kind != String || text.empty()) throw std::runtime_error("expected a nonempty string");
        return text;
    }
    bool asBool() const {
        if (kind != Bool) throw std::runtime_error("expected a boolean");
        return b;
    }
};

class Reader {
public:
    explicit Reader(const std::string& s) : s_(s) {}
    Node document() {
        Node n = value(0);
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        if (n.kind != Node::Object) fail("top level must be an object");
        return n;
    }

private:
    const std::string& s_;
    size_t i_ = 0;

    [[noreturn]] void fail(const char* what) const {
        throw std::runtime_error(std::string("JSON error at offset ") + std::to_string(i_) + ": " + what);
    }
    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
    }
    char peek() {
        ws();
        return i_ < s_.size() ? s_[i_] : '\0';
    }
    void expect(char c) {
        if (peek() != c) fail("unexpected character");
        ++i_;
    }
    static void utf8(std::string& out, unsigned cp) {
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
    }
    std::string str() {
        expect('"');
        std::string out;
        for (;;) {
            if (i_ >= s_.size()) fail("unterminated string");
            const unsigned char c = (unsigned char)s_[i_++];
            if (c == '"') return out;
            if (c < 0x20) fail("control character in string");
            if (c != '\\') {
                out += (char)c;
                continue;
            }
            if (i_ >= s_.size()) fail("bad escape");
            const char e = s_[i_++];
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
                    if (i_ + 4 > s_.size()) fail("short \\u escape");
                    unsigned cp = 0;
                    for (int k = 0; k < 4; ++k) {
                        const char h = s_[i_++];
                        cp <<= 4;
                        if (h >= '0' && h <= '9') cp |= (unsigned)(h - '0');
                        else if (h >= 'a' && h <= 'f') cp |= (unsigned)(h - 'a' + 10);
                        else if (h >= 'A' && h <= 'F') cp |= (unsigned)(h - 'A' + 10);
                        else fail("bad hex digit");
                    }
                    utf8(out, cp);
                    break;
                }
                default: fail("bad escape");
            }
        }
    }
    bool digit() const { return i_ < s_.size() && s_[i_] >= '0' && s_[i_] <= '9'; }
    Node number() {
        const size_t start = i_;
        if (s_[i_] == '-') ++i_;
        if (!digit()) fail("bad number");
        if (s_[i_] == '0') ++i_;
        else while (digit()) ++i_;
        if (i_ < s_.size() && s_[i_] == '.') {
            ++i_;
            if (!digit()) fail("bad fraction");
            while (digit()) ++i_;
        }
        if (i_ < s_.size() && (s_[i_] == 'e' || s_[i_] == 'E')) {
            ++i_;
            if (i_ < s_.size() && (s_[i_] == '+' || s_[i_] == '-')) ++i_;
            if (!digit()) fail("bad exponent");
            while (digit()) ++i_;
        }
        Node n;
        n.kind = Node::Number;
        n.text = s_.substr(start, i_ - start);
        return n;
    }
    bool literal(const char* word) {
        const size_t len = std::char_traits<char>::length(word);
        if (s_.compare(i_, len, word) != 0) return false;
        i_ += len;
        return true;
    }
    Node value(int depth) {
        if (depth > 64) fail("nesting too deep");
        const char c = peek();
        Node n;
        if (c == '{') {
            ++i_;
            n.kind = Node::Object;
            if (peek() == '}') { ++i_; return n; }
            for (;;) {
                if (peek() != '"') fail("expected key");
                std::string key = str();
                expect(':');
                if (n.members.count(key)) fail("duplicate key");
                n.members.emplace(std::move(key), value(depth + 1));
                const char d = peek();
                ++i_;
                if (d == '}') return n;
                if (d != ',') fail("expected , or }");
            }
        }
        if (c == '[') {
            ++i_;
            n.kind = Node::Array;
            if (peek() == ']') { ++i_; return n; }
            for (;;) {
                n.items.push_back(value(depth + 1));
                const char d = peek();
                ++i_;
                if (d == ']') return n;
                if (d != ',') fail("expected , or ]");
            }
        }
        if (c == '"') {
            n.kind = Node::String;
            n.text = str();
            return n;
        }
        if (c == '-' || (c >= '0' && c <= '9')) return number();
        if (literal("true")) { n.kind = Node::Bool; n.b = true; return n; }
        if (literal("false")) { n.kind = Node::Bool; n.b = false; return n; }
        if (literal("null")) { n.kind = Node::Null; return n; }
        fail("unexpected token");
    }
};

inline Node parse(const std::string& text) { return Reader(text).document(); }

}  // namespace json
}  // namespace bfly
