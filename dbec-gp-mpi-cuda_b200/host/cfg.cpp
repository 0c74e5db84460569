// cfg.cpp -- see cfg.h.
#include "cfg.h"

#include <cstdio>
#include <cstring>

namespace gpecli {

namespace {
constexpr int kMaxKeys = 256;
constexpr int kMaxLen = 256;
int g_size = 0;
char g_key[kMaxKeys][kMaxLen];
char g_val[kMaxKeys][kMaxLen];
}  // namespace

int cfg_init(const char *path) {
   FILE *f = std::fopen(path, "r");
   if (!f) return 0;
   g_size = 0;
   char buf[kMaxLen];
   // fgets with a 256-byte buffer, as cfg.c:42; field widths bound the copies
   // to the table entries (the reference's unbounded %s would overflow).
   while (std::fgets(buf, kMaxLen, f) != nullptr) {
      if (g_size >= kMaxKeys) break;
      if (std::sscanf(buf, "%255s = %255s", g_key[g_size], g_val[g_size]) == 2) g_size++;
   }
   std::fclose(f);
   return g_size;
}

const char *cfg_read(const char *key) {
   for (int i = 0; i < g_size; i++)
      if (!std::strcmp(key, g_key[i])) return g_val[i];
   return nullptr;
}

}  // namespace gpecli
