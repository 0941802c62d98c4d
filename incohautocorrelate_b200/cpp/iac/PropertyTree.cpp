// PropertyTree.cpp -- minimal XML reader/writer for the reference's
// property-tree files (see PropertyTree.h).
#include "PropertyTree.h"

#include <cctype>
#include <fstream>
#include <stdexcept>

namespace iac {

namespace {

std::string decode(const std::string &s)
{
    std::string o;
    for (size_t i = 0; i < s.size(); i++) {
        if (s[i] == '&') {
            const size_t e = s.find(';', i);
            if (e != std::string::npos) {
                const std::string ent = s.substr(i + 1, e - i - 1);
                if (ent == "lt") o += '<';
                else if (ent == "gt") o += '>';
                else if (ent == "amp") o += '&';
                else if (ent == "quot") o += '"';
                else if (ent == "apos") o += '\'';
                else o += s.substr(i, e - i + 1);
                i = e;
                continue;
            }
        }
        o += s[i];
    }
    return o;
}

std::string encode(const std::string &s)
{
    std::string o;
    for (char c : s) {
        if (c == '<') o += "&lt;";
        else if (c == '>') o += "&gt;";
        else if (c == '&') o += "&amp;";
        else o += c;
    }
    return o;
}

std::string trim(const std::string &s)
{
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) a++;
    while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
    return s.substr(a, b - a);
}

struct Parser {
    const std::string &x;
    size_t i = 0;
    explicit Parser(const std::string &s) : x(s) {}

    [[noreturn]] void fail(const char *what)
    {
        throw std::runtime_error(std::string("XML parse error: ") + what + " at offset " + std::to_string(i));
    }
    void skip_misc()
    {
        for (;;) {
            while (i < x.size() && std::isspace((unsigned char)x[i])) i++;
            if (x.compare(i, 4, "<!--") == 0) {
                const size_t e = x.find("-->", i);
                if (e == std::string::npos) fail("unterminated comment");
                i = e + 3;
            } else if (x.compare(i, 2, "<?") == 0) {
                const size_t e = x.find("?>", i);
                if (e == std::string::npos) fail("unterminated declaration");
                i = e + 2;
            } else {
                return;
            }
        }
    }
    PropertyTree element()
    {
        skip_misc();
        if (i >= x.size() || x[i] != '<') fail("expected '<'");
        i++;
        size_t s = i;
        while (i < x.size() && !std::isspace((unsigned char)x[i]) && x[i] != '>' && x[i] != '/') i++;
        PropertyTree n;
        n.name = x.substr(s, i - s);
        while (i < x.size() && x[i] != '>' && x[i] != '/') i++;  // attributes are ignored
        if (i < x.size() && x[i] == '/') {
            i += 2;
            return n;
        }
        i++;  // '>'
        std::string text;
        for (;;) {
            if (i >= x.size()) fail("unterminated element");
            if (x.compare(i, 4, "<!--") == 0) {
                skip_misc();
                continue;
            }
            if (x.compare(i, 2, "</") == 0) {
                const size_t e = x.find('>', i);
                if (e == std::string::npos) fail("unterminated end tag");
                if (trim(x.substr(i + 2, e - i - 2)) != n.name) fail("mismatched end tag");
                i = e + 1;
                break;
            }
            if (x[i] == '<') {
                n.children.push_back(element());
                continue;
            }
            text += x[i++];
        }
        n.text = decode(n.children.empty() ? text : trim(text));
        return n;
    }
};

void write(const PropertyTree &n, std::string &o)
{
    o += "<" + n.name + ">";
    if (n.children.empty()) {
        o += encode(n.text);
    } else {
        for (const auto &c : n.children) write(c, o);
    }
    o += "</" + n.name + ">";
}

}  // namespace

PropertyTree PropertyTree::ParseXml(const std::string &xml)
{
    Parser p(xml);
    PropertyTree doc;
    p.skip_misc();
    while (p.i < xml.size()) {
        doc.children.push_back(p.element());
        p.skip_misc();
    }
    return doc;
}

PropertyTree PropertyTree::ReadXml(const std::string &filename)
{
    std::ifstream f(filename, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + filename);
    std::stringstream ss;
    ss << f.rdbuf();
    return ParseXml(ss.str());
}

std::string PropertyTree::ToXml() const
{
    std::string o = "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n";
    for (const auto &c : children) write(c, o);
    o += "\n";
    return o;
}

void PropertyTree::WriteXml(const std::string &filename) const
{
    std::ofstream f(filename, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + filename);
    f << ToXml();
}

const PropertyTree *PropertyTree::Find(const std::string &path) const
{
    const PropertyTree *n = this;
    size_t s = 0;
    while (s <= path.size()) {
        const size_t e = path.find('.', s);
        const std::string part = path.substr(s, e == std::string::npos ? std::string::npos : e - s);
        const PropertyTree *next = nullptr;
        for (const auto &c : n->children)
            if (c.name == part) {
                next = &c;
                break;
            }
        if (!next) return nullptr;
        n = next;
        if (e == std::string::npos) break;
        s = e + 1;
    }
    return n;
}

PropertyTree &PropertyTree::Put(const std::string &path, const std::string &value)
{
    PropertyTree *n = this;
    size_t s = 0;
    for (;;) {
        const size_t e = path.find('.', s);
        const std::string part = path.substr(s, e == std::string::npos ? std::string::npos : e - s);
        PropertyTree *next = nullptr;
        for (auto &c : n->children)
            if (c.name == part) {
                next = &c;
                break;
            }
        if (!next) {
            n->children.push_back(PropertyTree());
            n->children.back().name = part;
            next = &n->children.back();
        }
        n = next;
        if (e == std::string::npos) break;
        s = e + 1;
    }
    n->text = value;
    return *n;
}

std::string PropertyTree::Get(const std::string &path, const std::string &fallback) const
{
    const PropertyTree *n = Find(path);
    return n ? n->text : fallback;
}

bool PropertyTree::GetBool(const std::string &path, bool fallback) const
{
    const PropertyTree *n = Find(path);
    if (!n) return fallback;
    const std::string t = trim(n->text);
    if (t == "true" || t == "1") return true;
    if (t == "false" || t == "0") return false;
    return fallback;
}

}  // namespace iac
