/* Stand-in for the time helper header Applications/Candidates.C includes
 * and the reference tree does not ship; Candidates.C uses nothing from it
 * (its own str2utctm covers the time parsing).  Test infrastructure. */
#pragma once
