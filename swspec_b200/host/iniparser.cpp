// iniparser.cpp -- INI reader with the reference's semantics
// (src/IniParser.cpp:48-265): every whitespace character is removed, any of
// / ' # starts a comment anywhere on a line, "[name]" opens a section,
// "key=value" (key of at least two characters) adds an entry, a duplicate
// key keeps the first value, integers are read through atof.
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <strings.h>

#include "sws_host.h"

namespace swshost {

namespace {

// What one line of the file holds once the parsing rules are applied.
enum class LineKind { Empty, Section, Entry, Malformed };

struct ParsedLine {
   LineKind kind = LineKind::Empty;
   std::string a, b;  // section name, or key and value
};

// The reference's rules, applied in order: drop every whitespace character,
// cut at the first comment character, then "[name]..." is a section header
// (non-empty name), "kk...=value" an entry (key of two or more characters).
ParsedLine classify(const std::string &raw)
{
   std::string t;
   t.reserve(raw.size());
   for (char ch : raw) {
      if (ch == '/' || ch == '\'' || ch == '#') break;
      if (!std::isspace(static_cast<unsigned char>(ch))) t.push_back(ch);
   }
   ParsedLine pl;
   if (t.empty()) return pl;
   if (t.front() == '[') {
      const size_t close = t.find(']');
      if (close != std::string::npos && close >= 2) {
         pl.kind = LineKind::Section;
         pl.a = t.substr(1, close - 1);
      } else {
         pl.kind = LineKind::Malformed;
      }
      return pl;
   }
   const size_t eq = t.find('=');
   if (eq != std::string::npos && eq >= 2) {
      pl.kind = LineKind::Entry;
      pl.a = t.substr(0, eq);
      pl.b = t.substr(eq + 1);
      return pl;
   }
   pl.kind = LineKind::Malformed;
   pl.a = t;
   return pl;
}

}  // namespace

IniParser::IniParser(const std::string &filename)
{
   std::ifstream in(filename.c_str());
   if (!in) {
      std::cerr << "INI file '" << filename << "' cannot be opened" << std::endl;
      return;
   }
   opened_ = true;
   std::string raw;
   for (int number = 0; std::getline(in, raw); number++) {
      const ParsedLine pl = classify(raw);
      switch (pl.kind) {
      case LineKind::Empty:
         break;
      case LineKind::Section:
         sections_.push_back(Section{pl.a, {}});
         section_index_ = (int)sections_.size() - 1;
         break;
      case LineKind::Entry:
         if (section_index_ < 0) break;  // entries before the first section are dropped
         if (hasKey(pl.a)) {
            std::cerr << "INI key '" << pl.a << "' repeated in section '" << sections_[section_index_].name
                      << "': the first value stays, '" << pl.b << "' is ignored" << std::endl;
            break;
         }
         sections_[section_index_].entries.push_back(KV{pl.a, pl.b});
         break;
      case LineKind::Malformed:
         std::cerr << "INI line " << number << " ignored (neither a [section] nor key=value): '" << raw << "'"
                   << std::endl;
         break;
      }
   }
}

bool IniParser::selectSection(const std::string &name)
{
   for (size_t i = 0; i < sections_.size(); i++)
      if (sections_[i].name == name) {
         section_index_ = (int)i;
         return true;
      }
   section_index_ = -1;
   return false;
}

bool IniParser::hasKey(const std::string &key) const
{
   if (section_index_ < 0) return false;
   for (const KV &kv : sections_[section_index_].entries)
      if (kv.key == key) return true;
   return false;
}

bool IniParser::getKeyValue(const char *key, std::string &value) const
{
   if (section_index_ < 0) return false;
   for (const KV &kv : sections_[section_index_].entries)
      if (kv.key == key) {
         value = kv.value;
         return true;
      }
   return false;
}

bool IniParser::getKeyValue(const char *key, int &value) const
{
   std::string s;
   if (!getKeyValue(key, s)) return false;
   value = (int)atof(s.c_str());
   return true;
}

bool IniParser::getKeyValue(const char *key, size_t &value) const
{
   int v;
   if (!getKeyValue(key, v)) return false;
   value = (size_t)v;
   return true;
}

bool IniParser::getKeyValue(const char *key, float &value) const
{
   std::string s;
   if (!getKeyValue(key, s)) return false;
   value = (float)atof(s.c_str());
   return true;
}

bool IniParser::getKeyValue(const char *key, bool &value) const
{
   std::string s;
   if (!getKeyValue(key, s)) return false;
   value = parse_YesNo(s.c_str());
   return true;
}

// Helpers::parse_YesNo (src/Helpers.cpp:69-79)
bool parse_YesNo(const char *str)
{
   if (strcasecmp(str, "yes") == 0 || strcasecmp(str, "true") == 0) return true;
   if (strcasecmp(str, "no") == 0 || strcasecmp(str, "false") == 0) return false;
   std::cerr << "Warning: Setting should be yes/no or true/false. Instead we got '" << str << std::endl;
   return false;
}

// Helpers::parse_Windowing (src/Helpers.cpp:87-104), plus BlackmanHarris
WindowFunctionType parse_Windowing(const char *str)
{
   if (strcasecmp(str, "None") == 0) return None;
   if (strcasecmp(str, "Cosine") == 0) return Cosine;
   if (strcasecmp(str, "Cosine2") == 0) return Cosine2;
   if (strcasecmp(str, "Hamming") == 0) return Hamming;
   if (strcasecmp(str, "Hann") == 0) return Hann;
   if (strcasecmp(str, "Blackman") == 0) return Blackman;
   if (strcasecmp(str, "BlackmanHarris") == 0) return BlackmanHarris;
   std::cerr << "Warning: window func  '" << str << "' not supported, will use Cosine2 instead." << std::endl;
   return Cosine2;
}

// Helpers::gcd (src/Helpers.cpp:150-162)
long long gcd(long long a, long long b)
{
   while (true) {
      a = a % b;
      if (a == 0) return b;
      b = b % a;
      if (b == 0) return a;
   }
}

}  // namespace swshost
