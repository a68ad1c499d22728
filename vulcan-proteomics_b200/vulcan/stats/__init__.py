"""Target-decoy statistics used to judge a search's output (reference ``vulcan/stats``)."""
