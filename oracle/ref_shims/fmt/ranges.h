/* Empty stand-in: the reference includes it but formats no ranges on the
 * build path (oracle compile only). */
#pragma once
#include "core.h"
