/* Empty stand-in for the MSVC <tchar.h> that the reference includes; the
   oracle build of the reference's CPU functions uses nothing from it. */
#pragma once
