/* Empty stand-in: the built-in index variables come from qmb_ref_shim.h. */
#pragma once
