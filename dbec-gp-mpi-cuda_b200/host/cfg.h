// cfg.h -- parameter-file reader with the semantics of the reference's
// cfg_init/cfg_read (src/utils/cfg.c:34-63, src/utils/cfg.h:37-41): lines are
// read in chunks of at most 255 characters and kept when sscanf("%s = %s")
// matches two fields; at most 256 keys; the first occurrence of a key wins.
#pragma once

namespace gpecli {

// Returns the number of keys read; 0 means "Wrong input parameter file."
// (a missing file or a file with no key = value line).
int cfg_init(const char *path);
// Value of key, or nullptr when absent.
const char *cfg_read(const char *key);

}  // namespace gpecli
