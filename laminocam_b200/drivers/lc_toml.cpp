// TOML subset parser (see lc_toml.hpp for the supported grammar).
#include "lc_toml.hpp"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace lc::toml {
namespace {

class Parser {
  public:
    Parser(const std::string &text, const std::string &name) : t_(text), name_(name) {}

    Table run() {
        Table root;
        Table *cur = &root;
        for (;;) {
            skip_ws_lines();
            if (eof()) break;
            if (peek() == '[') {
                const bool aot = peek(1) == '[';
                pos_ += aot ? 2 : 1;
                skip_inline_ws();
                std::vector<std::string> path = key_path();
                skip_inline_ws();
                expect(']');
                if (aot) expect(']');
                end_of_line();
                cur = aot ? open_array_table(root, path) : open_table(root, path);
            } else {
                std::vector<std::string> path = key_path();
                skip_inline_ws();
                expect('=');
                skip_inline_ws();
                Value v = value();
                end_of_line();
                assign(*cur, path, std::move(v));
            }
        }
        return root;
    }

  private:
    [[noreturn]] void fail(const std::string &msg) const {
        throw std::runtime_error(name_ + ":" + std::to_string(line_) + ": " + msg);
    }
    bool eof() const { return pos_ >= t_.size(); }
    char peek(size_t k = 0) const { return pos_ + k < t_.size() ? t_[pos_ + k] : '\0'; }
    char get() {
        char c = peek();
        ++pos_;
        if (c == '\n') ++line_;
        return c;
    }
    void expect(char c) {
        if (peek() != c) fail(std::string("expected '") + c + "'");
        get();
    }
    void skip_inline_ws() {
        while (peek() == ' ' || peek() == '\t') get();
    }
    void skip_comment() {
        if (peek() == '#')
            while (!eof() && peek() != '\n') get();
    }
    // whitespace, newlines and comments
    void skip_ws_lines() {
        for (;;) {
            skip_inline_ws();
            if (peek() == '#') skip_comment();
            if (peek() == '\r' || peek() == '\n') {
                get();
                continue;
            }
            break;
        }
    }
    void end_of_line() {
        skip_inline_ws();
        skip_comment();
        if (peek() == '\r') get();
        if (!eof() && peek() != '\n') fail("unexpected text after a value");
    }

    std::string bare_or_quoted_key() {
        if (peek() == '"') return basic_string();
        if (peek() == '\'') return literal_string();
        std::string k;
        while (std::isalnum((unsigned char)peek()) || peek() == '_' || peek() == '-') k += get();
        if (k.empty()) fail("expected a key");
        return k;
    }
    std::vector<std::string> key_path() {
        std::vector<std::string> p{bare_or_quoted_key()};
        for (;;) {
            skip_inline_ws();
            if (peek() != '.') break;
            get();
            skip_inline_ws();
            p.push_back(bare_or_quoted_key());
        }
        return p;
    }

    std::string basic_string() {
        expect('"');
        if (peek() == '"' && peek(1) == '"') fail("multi-line strings are not supported");
        std::string s;
        for (;;) {
            if (eof() || peek() == '\n') fail("unterminated string");
            char c = get();
            if (c == '"') break;
            if (c != '\\') {
                s += c;
                continue;
            }
            char e = get();
            switch (e) {
                case 'n': s += '\n'; break;
                case 't': s += '\t'; break;
                case 'r': s += '\r'; break;
                case 'b': s += '\b'; break;
                case 'f': s += '\f'; break;
                case '"': s += '"'; break;
                case '\\': s += '\\'; break;
                case 'u':
                case 'U': {
                    const int n = e == 'u' ? 4 : 8;
                    std::string hex;
                    for (int k = 0; k < n; ++k) hex += get();
                    unsigned long cp = std::strtoul(hex.c_str(), nullptr, 16);
                    append_utf8(s, cp);
                    break;
                }
                default: fail("unknown escape in string");
            }
        }
        return s;
    }
    static void append_utf8(std::string &s, unsigned long cp) {
        if (cp < 0x80) {
            s += (char)cp;
        } else if (cp < 0x800) {
            s += (char)(0xC0 | (cp >> 6));
            s += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            s += (char)(0xE0 | (cp >> 12));
            s += (char)(0x80 | ((cp >> 6) & 0x3F));
            s += (char)(0x80 | (cp & 0x3F));
        } else {
            s += (char)(0xF0 | (cp >> 18));
            s += (char)(0x80 | ((cp >> 12) & 0x3F));
            s += (char)(0x80 | ((cp >> 6) & 0x3F));
            s += (char)(0x80 | (cp & 0x3F));
        }
    }
    std::string literal_string() {
        expect('\'');
        if (peek() == '\'' && peek(1) == '\'') fail("multi-line strings are not supported");
        std::string s;
        for (;;) {
            if (eof() || peek() == '\n') fail("unterminated string");
            char c = get();
            if (c == '\'') break;
            s += c;
        }
        return s;
    }

    Value value() {
        Value v;
        const char c = peek();
        if (c == '"') {
            v.kind = Value::STRING;
            v.s = basic_string();
        } else if (c == '\'') {
            v.kind = Value::STRING;
            v.s = literal_string();
        } else if (c == '[') {
            v = array();
        } else if (c == '{') {
            v = inline_table();
        } else if (t_.compare(pos_, 4, "true") == 0) {
            pos_ += 4;
            v.kind = Value::BOOL;
            v.b = true;
        } else if (t_.compare(pos_, 5, "false") == 0) {
            pos_ += 5;
            v.kind = Value::BOOL;
            v.b = false;
        } else {
            v = number();
        }
        return v;
    }

    Value number() {
        std::string tok;
        while (!eof()) {
            char c = peek();
            if (std::isalnum((unsigned char)c) || c == '+' || c == '-' || c == '.' || c == '_' ||
                c == ':')
                tok += get();
            else
                break;
        }
        if (tok.empty()) fail("expected a value");
        if (tok.find(':') != std::string::npos || (tok.size() >= 10 && tok[4] == '-' && tok[7] == '-'))
            fail("dates and times are not supported");
        std::string clean;
        for (size_t k = 0; k < tok.size(); ++k) {
            if (tok[k] == '_') {
                if (k == 0 || k + 1 == tok.size() || !std::isalnum((unsigned char)tok[k - 1]) ||
                    !std::isalnum((unsigned char)tok[k + 1]))
                    fail("misplaced '_' in a number");
                continue;
            }
            clean += tok[k];
        }
        Value v;
        std::string body = clean;
        int sign = 1;
        if (!body.empty() && (body[0] == '+' || body[0] == '-')) {
            sign = body[0] == '-' ? -1 : 1;
            body = body.substr(1);
        }
        if (body == "inf" || body == "nan") {
            v.kind = Value::FLOAT;
            v.f = body == "inf" ? sign * HUGE_VAL : std::nan("");
            return v;
        }
        if (body.size() > 2 && body[0] == '0' && (body[1] == 'x' || body[1] == 'o' || body[1] == 'b')) {
            if (sign < 0 || clean[0] == '+') fail("signed non-decimal integer");
            const int base = body[1] == 'x' ? 16 : (body[1] == 'o' ? 8 : 2);
            char *end = nullptr;
            v.kind = Value::INT;
            v.i = (int64_t)std::strtoull(body.c_str() + 2, &end, base);
            if (*end) fail("bad integer '" + tok + "'");
            return v;
        }
        const bool is_float = body.find_first_of(".eE") != std::string::npos;
        char *end = nullptr;
        if (is_float) {
            v.kind = Value::FLOAT;
            v.f = std::strtod(clean.c_str(), &end);
        } else {
            if (body.size() > 1 && body[0] == '0') fail("leading zero in integer '" + tok + "'");
            v.kind = Value::INT;
            v.i = (int64_t)std::strtoll(clean.c_str(), &end, 10);
        }
        if (end == nullptr || *end) fail("bad number '" + tok + "'");
        return v;
    }

    Value array() {
        expect('[');
        Value v = Value::array();
        for (;;) {
            skip_ws_lines();
            if (peek() == ']') {
                get();
                break;
            }
            v.arr->push_back(value());
            skip_ws_lines();
            if (peek() == ',') {
                get();
                continue;
            }
            skip_ws_lines();
            expect(']');
            break;
        }
        return v;
    }

    Value inline_table() {
        expect('{');
        Value v = Value::table();
        skip_inline_ws();
        if (peek() == '}') {
            get();
            return v;
        }
        for (;;) {
            skip_inline_ws();
            std::vector<std::string> path = key_path();
            skip_inline_ws();
            expect('=');
            skip_inline_ws();
            assign(*v.tbl, path, value());
            skip_inline_ws();
            if (peek() == ',') {
                get();
                continue;
            }
            expect('}');
            break;
        }
        return v;
    }

    // walks/creates the intermediate tables of a dotted path
    Table *descend(Table &root, const std::vector<std::string> &path, size_t upto) {
        Table *t = &root;
        for (size_t k = 0; k < upto; ++k) {
            auto it = t->find(path[k]);
            if (it == t->end()) it = t->emplace(path[k], Value::table()).first;
            Value &v = it->second;
            if (v.is_table()) {
                t = v.tbl.get();
            } else if (v.is_array() && v.table_array && !v.arr->empty()) {
                t = v.arr->back().tbl.get();
            } else {
                fail("key '" + path[k] + "' is not a table");
            }
        }
        return t;
    }
    Table *open_table(Table &root, const std::vector<std::string> &path) {
        Table *parent = descend(root, path, path.size() - 1);
        auto it = parent->find(path.back());
        if (it == parent->end()) it = parent->emplace(path.back(), Value::table()).first;
        if (!it->second.is_table()) fail("[" + path.back() + "] redefines a value");
        return it->second.tbl.get();
    }
    Table *open_array_table(Table &root, const std::vector<std::string> &path) {
        Table *parent = descend(root, path, path.size() - 1);
        auto it = parent->find(path.back());
        if (it == parent->end()) {
            Value a = Value::array();
            a.table_array = true;
            it = parent->emplace(path.back(), a).first;
        }
        if (!it->second.is_array() || !it->second.table_array)
            fail("[[" + path.back() + "]] redefines a value");
        it->second.arr->push_back(Value::table());
        return it->second.arr->back().tbl.get();
    }
    void assign(Table &t, const std::vector<std::string> &path, Value v) {
        Table *parent = descend(t, path, path.size() - 1);
        if (parent->count(path.back())) fail("duplicate key '" + path.back() + "'");
        parent->emplace(path.back(), std::move(v));
    }

    const std::string &t_;
    std::string name_;
    size_t pos_ = 0;
    int line_ = 1;
};

}  // namespace

Table parse(const std::string &text, const std::string &name) { return Parser(text, name).run(); }

Table parse_file(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("TOML file does not exist: " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return parse(ss.str(), path);
}

const Value *find(const Table &t, const std::string &key) {
    auto it = t.find(key);
    return it == t.end() ? nullptr : &it->second;
}

const Table *find_table(const Table &t, const std::string &key) {
    const Value *v = find(t, key);
    return v && v->is_table() ? v->tbl.get() : nullptr;
}

}  // namespace lc::toml
