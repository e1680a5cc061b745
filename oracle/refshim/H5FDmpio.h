/* Stand-in: intentionally empty. */
