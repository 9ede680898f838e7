// iniparser.cpp -- INI reader with the reference's semantics
// (src/IniParser.cpp:48-265): every whitespace character is removed, any of
// / ' # starts a comment anywhere on a line, "[name]" opens a section,
// "key=value" (key of at least two characters) adds an entry, a duplicate
// key keeps the first value, integers are read through atof.
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <strings.h>

#include "sws_host.h"

namespace swshost {

IniParser::IniParser(const std::string &filename)
{
   std::ifstream file(filename.c_str());
   if (!file.is_open()) {
      std::cerr << "Error: Could not open INI file " << filename << std::endl;
      return;
   }
   opened_ = true;
   std::string line;
   int linenr = -1;
   while (!std::getline(file, line).fail()) {
      linenr++;
      std::string mline, element;
      std::istringstream istr(line);
      while (istr >> element) mline += element;
      size_t cpos = mline.find_first_of("/'#", 0);
      if (cpos != std::string::npos) mline.resize(cpos);
      if (mline.empty()) continue;
      if (mline[0] == '[') {
         cpos = mline.find_first_of("]", 0);
         if (cpos == std::string::npos || cpos <= 1) {
            std::cerr << "INI section line " << linenr << " '" << line << "' incorrectly formed'" << std::endl;
            continue;
         }
         Section sec;
         sec.name = mline.substr(1, cpos - 1);
         sections_.push_back(sec);
         section_index_ = (int)sections_.size() - 1;
         continue;
      }
      cpos = mline.find_first_of("=", 0);
      if (cpos != std::string::npos && cpos > 1) {
         if (section_index_ < 0) continue;
         KV kv;
         kv.key = mline.substr(0, cpos);
         kv.value = mline.substr(cpos + 1);
         if (hasKey(kv.key)) {
            std::cerr << "Warning: INI section contains duplicate key '" << kv.key << "'! "
                      << "Not assigning new value '" << kv.value << "'." << std::endl;
            continue;
         }
         sections_[section_index_].entries.push_back(kv);
         continue;
      }
      std::cerr << "INI has malformed line " << linenr << " '" << line << "' (parsed as '" << mline << "') "
                << std::endl;
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
