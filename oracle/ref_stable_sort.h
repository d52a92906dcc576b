// TEST INFRASTRUCTURE ONLY.  Pre-included (g++ -include) into the reference sources of
// the pinning build: every standard header is included first, then the token `sort`
// is mapped to `stable_sort`, so sort_iota_by_key (opp_lib/include/opp_util.h:211-221)
// orders equal cell indices by particle index.  The reference sources are not modified.
#pragma once
#include <bits/stdc++.h>
#define sort stable_sort
