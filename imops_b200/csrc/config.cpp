// config.cpp -- TOML-subset and JSON parsers for pipeline configs.
#include "config.hpp"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <sstream>

namespace imops {
namespace cfg {

namespace {

struct Cursor {
    const std::string& s;
    size_t p = 0;
    int line = 1;
    explicit Cursor(const std::string& str) : s(str) {}
    bool eof() const { return p >= s.size(); }
    char peek(size_t o = 0) const { return p + o < s.size() ? s[p + o] : '\0'; }
    char get() {
        char c = s[p++];
        if (c == '\n') line++;
        return c;
    }
};

std::string where(const Cursor& c) { return " (line " + std::to_string(c.line) + ")"; }

void append_utf8(std::string& out, unsigned cp) {
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

bool read_escaped(Cursor& c, char quote, std::string* out, std::string* err) {
    // opening quote consumed
    while (!c.eof()) {
        char ch = c.get();
        if (ch == quote) return true;
        if (ch == '\n' && quote == '"') {
            *err = "newline in string" + where(c);
            return false;
        }
        if (ch == '\\') {
            if (c.eof()) break;
            char e = c.get();
            switch (e) {
                case '"': *out += '"'; break;
                case '\\': *out += '\\'; break;
                case '/': *out += '/'; break;
                case 'b': *out += '\b'; break;
                case 'f': *out += '\f'; break;
                case 'n': *out += '\n'; break;
                case 'r': *out += '\r'; break;
                case 't': *out += '\t'; break;
                case 'u': case 'U': {
                    int nd = e == 'u' ? 4 : 8;
                    unsigned cp = 0;
                    for (int k = 0; k < nd; k++) {
                        if (c.eof() || !std::isxdigit((unsigned char)c.peek())) {
                            *err = "bad unicode escape" + where(c);
                            return false;
                        }
                        char h = c.get();
                        cp = cp * 16 + (unsigned)(std::isdigit((unsigned char)h) ? h - '0' : (std::tolower(h) - 'a' + 10));
                    }
                    append_utf8(*out, cp);
                    break;
                }
                default:
                    *err = std::string("bad escape \\") + e + where(c);
                    return false;
            }
        } else {
            *out += ch;
        }
    }
    *err = "unterminated string" + where(c);
    return false;
}

bool read_number(Cursor& c, Value* v, std::string* err, bool toml) {
    size_t start = c.p;
    std::string num;
    if (c.peek() == '+' || c.peek() == '-') num += c.get();
    if (toml && (c.s.compare(c.p, 3, "inf") == 0 || c.s.compare(c.p, 3, "nan") == 0)) {
        std::string w = c.s.substr(c.p, 3);
        c.p += 3;
        v->kind = Value::FLOAT;
        v->f = w == "inf" ? INFINITY : NAN;
        if (!num.empty() && num[0] == '-') v->f = -v->f;
        return true;
    }
    bool is_float = false;
    while (!c.eof()) {
        char ch = c.peek();
        if (std::isdigit((unsigned char)ch)) {
            num += c.get();
        } else if (toml && ch == '_') {
            c.get();
        } else if (ch == '.' || ch == 'e' || ch == 'E') {
            is_float = true;
            num += c.get();
            if ((ch == 'e' || ch == 'E') && (c.peek() == '+' || c.peek() == '-')) num += c.get();
        } else {
            break;
        }
    }
    if (num.empty() || num == "+" || num == "-") {
        *err = "expected a value" + where(c);
        c.p = start;
        return false;
    }
    char* end = nullptr;
    if (is_float) {
        v->kind = Value::FLOAT;
        v->f = std::strtod(num.c_str(), &end);
    } else {
        v->kind = Value::INT;
        v->i = std::strtoll(num.c_str(), &end, 10);
    }
    if (!end || *end != '\0') {
        *err = "malformed number '" + num + "'" + where(c);
        return false;
    }
    return true;
}

// ---- TOML ------------------------------------------------------------------

void toml_skip_ws(Cursor& c, bool newlines) {
    while (!c.eof()) {
        char ch = c.peek();
        if (ch == ' ' || ch == '\t' || ch == '\r' || (newlines && ch == '\n')) {
            c.get();
        } else if (ch == '#') {
            while (!c.eof() && c.peek() != '\n') c.get();
        } else {
            break;
        }
    }
}

bool toml_key(Cursor& c, std::string* key, std::string* err) {
    key->clear();
    if (c.peek() == '"') {
        c.get();
        return read_escaped(c, '"', key, err);
    }
    if (c.peek() == '\'') {
        c.get();
        while (!c.eof() && c.peek() != '\'') *key += c.get();
        if (c.eof()) {
            *err = "unterminated key" + where(c);
            return false;
        }
        c.get();
        return true;
    }
    while (!c.eof() && (std::isalnum((unsigned char)c.peek()) || c.peek() == '_' || c.peek() == '-')) *key += c.get();
    if (key->empty()) {
        *err = "expected a key" + where(c);
        return false;
    }
    return true;
}

bool toml_value(Cursor& c, Value* v, std::string* err);

bool toml_inline_table(Cursor& c, Value* v, std::string* err) {
    c.get();  // {
    v->kind = Value::TABLE;
    toml_skip_ws(c, false);
    if (c.peek() == '}') {
        c.get();
        return true;
    }
    for (;;) {
        toml_skip_ws(c, false);
        std::string k;
        if (!toml_key(c, &k, err)) return false;
        toml_skip_ws(c, false);
        if (c.peek() != '=') {
            *err = "expected '=' in inline table" + where(c);
            return false;
        }
        c.get();
        toml_skip_ws(c, false);
        Value item;
        if (!toml_value(c, &item, err)) return false;
        v->t.emplace_back(k, item);
        toml_skip_ws(c, false);
        if (c.peek() == ',') {
            c.get();
            continue;
        }
        if (c.peek() == '}') {
            c.get();
            return true;
        }
        *err = "expected ',' or '}' in inline table" + where(c);
        return false;
    }
}

bool toml_array(Cursor& c, Value* v, std::string* err) {
    c.get();  // [
    v->kind = Value::ARRAY;
    for (;;) {
        toml_skip_ws(c, true);
        if (c.peek() == ']') {
            c.get();
            return true;
        }
        Value item;
        if (!toml_value(c, &item, err)) return false;
        v->a.push_back(item);
        toml_skip_ws(c, true);
        if (c.peek() == ',') {
            c.get();
            continue;
        }
        if (c.peek() == ']') {
            c.get();
            return true;
        }
        *err = "expected ',' or ']' in array" + where(c);
        return false;
    }
}

bool toml_value(Cursor& c, Value* v, std::string* err) {
    char ch = c.peek();
    if (ch == '"') {
        c.get();
        v->kind = Value::STRING;
        return read_escaped(c, '"', &v->s, err);
    }
    if (ch == '\'') {
        c.get();
        v->kind = Value::STRING;
        while (!c.eof() && c.peek() != '\'') v->s += c.get();
        if (c.eof()) {
            *err = "unterminated string" + where(c);
            return false;
        }
        c.get();
        return true;
    }
    if (ch == '[') return toml_array(c, v, err);
    if (ch == '{') return toml_inline_table(c, v, err);
    if (c.s.compare(c.p, 4, "true") == 0) {
        c.p += 4;
        v->kind = Value::BOOL;
        v->b = true;
        return true;
    }
    if (c.s.compare(c.p, 5, "false") == 0) {
        c.p += 5;
        v->kind = Value::BOOL;
        v->b = false;
        return true;
    }
    return read_number(c, v, err, true);
}

// ---- JSON ------------------------------------------------------------------

void json_ws(Cursor& c) {
    while (!c.eof() && std::isspace((unsigned char)c.peek())) c.get();
}

bool json_value(Cursor& c, Value* v, std::string* err, int depth) {
    if (depth > 64) {
        *err = "nesting too deep";
        return false;
    }
    json_ws(c);
    char ch = c.peek();
    if (ch == '{') {
        c.get();
        v->kind = Value::TABLE;
        json_ws(c);
        if (c.peek() == '}') {
            c.get();
            return true;
        }
        for (;;) {
            json_ws(c);
            if (c.peek() != '"') {
                *err = "expected a string key" + where(c);
                return false;
            }
            c.get();
            std::string k;
            if (!read_escaped(c, '"', &k, err)) return false;
            json_ws(c);
            if (c.peek() != ':') {
                *err = "expected ':'" + where(c);
                return false;
            }
            c.get();
            Value item;
            if (!json_value(c, &item, err, depth + 1)) return false;
            v->t.emplace_back(k, item);
            json_ws(c);
            if (c.peek() == ',') {
                c.get();
                continue;
            }
            if (c.peek() == '}') {
                c.get();
                return true;
            }
            *err = "expected ',' or '}'" + where(c);
            return false;
        }
    }
    if (ch == '[') {
        c.get();
        v->kind = Value::ARRAY;
        json_ws(c);
        if (c.peek() == ']') {
            c.get();
            return true;
        }
        for (;;) {
            Value item;
            if (!json_value(c, &item, err, depth + 1)) return false;
            v->a.push_back(item);
            json_ws(c);
            if (c.peek() == ',') {
                c.get();
                continue;
            }
            if (c.peek() == ']') {
                c.get();
                return true;
            }
            *err = "expected ',' or ']'" + where(c);
            return false;
        }
    }
    if (ch == '"') {
        c.get();
        v->kind = Value::STRING;
        return read_escaped(c, '"', &v->s, err);
    }
    if (c.s.compare(c.p, 4, "true") == 0) {
        c.p += 4;
        v->kind = Value::BOOL;
        v->b = true;
        return true;
    }
    if (c.s.compare(c.p, 5, "false") == 0) {
        c.p += 5;
        v->kind = Value::BOOL;
        v->b = false;
        return true;
    }
    if (c.s.compare(c.p, 4, "null") == 0) {
        c.p += 4;
        v->kind = Value::NUL;
        return true;
    }
    return read_number(c, v, err, false);
}

void json_escape(std::ostringstream& o, const std::string& s) {
    o << '"';
    for (unsigned char ch : s) {
        switch (ch) {
            case '"': o << "\\\""; break;
            case '\\': o << "\\\\"; break;
            case '\n': o << "\\n"; break;
            case '\r': o << "\\r"; break;
            case '\t': o << "\\t"; break;
            default:
                if (ch < 0x20) {
                    char buf[8];
                    std::snprintf(buf, sizeof buf, "\\u%04x", ch);
                    o << buf;
                } else {
                    o << ch;
                }
        }
    }
    o << '"';
}

void to_json_rec(std::ostringstream& o, const Value& v) {
    switch (v.kind) {
        case Value::NUL: o << "null"; break;
        case Value::BOOL: o << (v.b ? "true" : "false"); break;
        case Value::INT: o << v.i; break;
        case Value::FLOAT: {
            if (!std::isfinite(v.f)) {
                o << "null";
            } else {
                char buf[64];
                std::snprintf(buf, sizeof buf, "%.17g", v.f);
                std::string s = buf;
                if (s.find_first_of(".eE") == std::string::npos) s += ".0";
                o << s;
            }
            break;
        }
        case Value::STRING: json_escape(o, v.s); break;
        case Value::ARRAY:
            o << '[';
            for (size_t k = 0; k < v.a.size(); k++) {
                if (k) o << ',';
                to_json_rec(o, v.a[k]);
            }
            o << ']';
            break;
        case Value::TABLE:
            o << '{';
            for (size_t k = 0; k < v.t.size(); k++) {
                if (k) o << ',';
                json_escape(o, v.t[k].first);
                o << ':';
                to_json_rec(o, v.t[k].second);
            }
            o << '}';
            break;
    }
}

}  // namespace

bool parse_toml(const std::string& text, Value* out, std::string* err) {
    Cursor c(text);
    out->kind = Value::TABLE;
    out->t.clear();
    Value* cur = out;
    for (;;) {
        toml_skip_ws(c, true);
        if (c.eof()) return true;
        if (c.peek() == '[') {
            bool arr = c.peek(1) == '[';
            c.get();
            if (arr) c.get();
            toml_skip_ws(c, false);
            std::string name;
            if (!toml_key(c, &name, err)) return false;
            toml_skip_ws(c, false);
            if (c.peek() != ']' || (arr && c.peek(1) != ']')) {
                *err = "malformed table header" + where(c);
                return false;
            }
            c.get();
            if (arr) c.get();
            Value* slot = out->get_mut(name);
            if (arr) {
                if (!slot) {
                    Value a;
                    a.kind = Value::ARRAY;
                    out->t.emplace_back(name, a);
                    slot = &out->t.back().second;
                } else if (slot->kind != Value::ARRAY) {
                    *err = "key '" + name + "' is not an array of tables" + where(c);
                    return false;
                }
                Value tbl;
                tbl.kind = Value::TABLE;
                slot->a.push_back(tbl);
                cur = &slot->a.back();
            } else {
                if (slot) {
                    *err = "duplicate table '" + name + "'" + where(c);
                    return false;
                }
                Value tbl;
                tbl.kind = Value::TABLE;
                out->t.emplace_back(name, tbl);
                cur = &out->t.back().second;
            }
            continue;
        }
        std::string key;
        if (!toml_key(c, &key, err)) return false;
        toml_skip_ws(c, false);
        if (c.peek() != '=') {
            *err = "expected '=' after key '" + key + "'" + where(c);
            return false;
        }
        c.get();
        toml_skip_ws(c, false);
        Value v;
        if (!toml_value(c, &v, err)) return false;
        if (cur->get(key)) {
            *err = "duplicate key '" + key + "'" + where(c);
            return false;
        }
        cur->t.emplace_back(key, v);
        toml_skip_ws(c, false);
        if (!c.eof() && c.peek() != '\n') {
            *err = "unexpected text after value of '" + key + "'" + where(c);
            return false;
        }
    }
}

bool parse_json(const std::string& text, Value* out, std::string* err) {
    Cursor c(text);
    if (!json_value(c, out, err, 0)) return false;
    json_ws(c);
    if (!c.eof()) {
        *err = "trailing characters after JSON value" + where(c);
        return false;
    }
    return true;
}

std::string to_json(const Value& v) {
    std::ostringstream o;
    to_json_rec(o, v);
    return o.str();
}

}  // namespace cfg
}  // namespace imops
